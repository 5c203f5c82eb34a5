"""The learned gate's pipeline: traces from the plain search, labels, device
training, thresholds.

The gate (include/rover_b200.h, ROVER_MODE_GATED) is a 5 -> 64 -> 64 -> 2 MLP
that the batched search consults per candidate (refine-needed: correct the
candidate with its residual row, or keep its ADC distance) and per step
(stop-expanding).  It is trained on rows that the plain search with full
correction writes (calculator_rover_pq_trace, the reference's expansion
order):

* refine rows -- every scored candidate and every shortlisted entry seed,
  labelled 1 when its corrected distance entered the pool;
* stop rows -- every expansion source, labelled 1 when all of the query's
  final top-k had already been scored before this expansion (so stopping here
  would have lost nothing).

Inputs per row: log quantized distance, pool rank / L, log worst pool
distance, hop count / L, query norm (the order the kernels use).
Training runs on the device (calculator_rover_gate_train).  Full correction
stays the fallback: without a loaded gate, ROVER_MODE_GATED runs as
ROVER_MODE_BATCHED.
"""
from __future__ import annotations

import json
from dataclasses import asdict, dataclass, field
from pathlib import Path

import numpy as np

from .calculator import Calculator

SOURCE, SEED, ENTERED = 2, 4, 1


def features(rows: np.ndarray, pool: int | np.ndarray) -> np.ndarray:
    """Raw gate inputs [n][5] of trace rows (pool: L per row or one L)."""
    L = np.asarray(pool, np.float32)
    hop = rows["hop"].astype(np.float32) / L
    return np.stack([np.log(np.maximum(rows["quantized"], 1e-30)), rows["rank"],
                     np.log(np.maximum(rows["worst"], 1e-30)), hop, rows["qnorm"]], 1).astype(np.float32)


def labels(rows: np.ndarray, ids: np.ndarray, counts: np.ndarray, top_k: int):
    """Targets y[n][2] and masks m[n][2] of trace rows, given the search's
    final results ids[nq][k] / counts[nq]."""
    nq = ids.shape[0]
    src = (rows["flags"] & SOURCE) != 0
    seed = (rows["flags"] & SEED) != 0
    q = rows["query"].astype(np.int64)
    # last hop at which a final result was scored (entry seeds count as -1)
    k = np.minimum(counts, top_k)
    res_q = np.repeat(np.arange(nq, dtype=np.int64), k)
    res_id = np.concatenate([ids[i, :k[i]] for i in range(nq)]).astype(np.int64) if nq else np.zeros(0, np.int64)
    span = np.int64(1) << 32
    res_key = np.sort(res_q * span + res_id)
    row_key = q * span + rows["id"].astype(np.int64)
    is_result = ~src & np.isin(row_key, res_key)
    hop_found = np.where(seed, -1, rows["hop"]).astype(np.int64)
    last = np.full(nq, -1, np.int64)
    np.maximum.at(last, q[is_result], hop_found[is_result])
    y = np.zeros((len(rows), 2), np.float32)
    m = np.zeros((len(rows), 2), np.float32)
    y[:, 0] = ((rows["flags"] & ENTERED) != 0) & ~src
    m[:, 0] = ~src
    y[:, 1] = src & (rows["hop"] > last[q])
    m[:, 1] = src
    return y, m


def bands(rows: np.ndarray, lo_quantile: float = 0.01, hi_quantile: float = 0.999) -> tuple[float, float]:
    """ADC / worst ratio band the MLP decides in: below band_lo almost no
    candidate stays out of the pool (corrected without asking), above band_hi
    almost none enters (kept at its ADC distance)."""
    cand = (rows["flags"] & SOURCE) == 0
    ratio = rows["quantized"][cand] / np.maximum(rows["worst"][cand], 1e-30)
    entered = (rows["flags"][cand] & ENTERED) != 0
    out = ratio[~entered]
    inn = ratio[entered]
    lo = float(np.quantile(out, lo_quantile)) if out.size else 0.0
    hi = float(np.quantile(inn, hi_quantile)) if inn.size else np.inf
    return lo, max(hi, lo)


@dataclass
class GateModel:
    params: np.ndarray
    mu: np.ndarray
    sigma: np.ndarray
    band_lo: float = 0.0
    band_hi: float = np.inf
    refine_logit: float = 0.0
    stop_logit: float = np.inf
    info: dict = field(default_factory=dict)

    def load(self, calc: Calculator, **override) -> None:
        t = dict(band_lo=self.band_lo, band_hi=self.band_hi, refine_logit=self.refine_logit,
                 stop_logit=self.stop_logit)
        t.update(override)
        calc.gate_load(self.params, self.mu, self.sigma, **t)

    def save(self, path: str | Path) -> None:
        path = Path(path)
        np.savez(path, params=self.params, mu=self.mu, sigma=self.sigma)
        meta = {k: v for k, v in asdict(self).items() if k not in ("params", "mu", "sigma")}
        path.with_suffix(".json").write_text(json.dumps(meta, default=float))

    @classmethod
    def open(cls, path: str | Path) -> "GateModel":
        path = Path(path)
        z = np.load(path if path.suffix == ".npz" else path.with_suffix(".npz"))
        meta = json.loads(path.with_suffix(".json").read_text())
        return cls(z["params"], z["mu"], z["sigma"], **meta)


def collect(calc: Calculator, queries: np.ndarray, pool: int, top_k: int = 10, chunk: int = 4096,
            rows_per_query: int = 4096, **search) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Trace rows of the plain search over `queries` (chunked), with query
    numbers made global; returns rows, final ids, counts."""
    all_rows, ids, counts = [], [], []
    for q0 in range(0, len(queries), chunk):
        qs = queries[q0:q0 + chunk]
        r = calc.pq_trace(qs, pool, capacity=len(qs) * rows_per_query, top_k=top_k, **search)
        if r["row_count"] > len(r["rows"]):
            raise RuntimeError(f"trace capacity {len(r['rows'])} below {r['row_count']} rows")
        rows = r["rows"].copy()
        rows["query"] += q0
        all_rows.append(rows)
        ids.append(r["ids"])
        counts.append(r["counts"])
    return np.concatenate(all_rows), np.concatenate(ids), np.concatenate(counts)


def train(calc: Calculator, rows: np.ndarray, ids: np.ndarray, counts: np.ndarray, pool: int, top_k: int = 10,
          max_rows: int = 5_000_000, epochs: int = 4, batch: int = 4096, lr: float = 2e-3, seed: int = 1,
          pos_weight=(1.0, 1.0)) -> GateModel:
    """Labels, subsampling to max_rows (stop rows always kept), device
    training.  Returns the model with its ADC band; thresholds are set by
    the caller's calibration."""
    y, m = labels(rows, ids, counts, top_k)
    x = features(rows, pool)
    n = len(rows)
    if n > max_rows:
        rng = np.random.default_rng(seed)
        src = (rows["flags"] & SOURCE) != 0
        keep = src | (rng.random(n) < (max_rows - src.sum()) / max(1, (~src).sum()))
        x, y, m = x[keep], y[keep], m[keep]
    out = calc.gate_train(x, y, m, epochs=epochs, batch=batch, lr=lr, seed=seed, pos_weight=pos_weight)
    lo, hi = bands(rows)
    info = dict(rows=int(len(x)), refine_rows=int(m[:, 0].sum()), refine_positive=float(y[m[:, 0] > 0, 0].mean()),
                stop_rows=int(m[:, 1].sum()), stop_positive=float(y[m[:, 1] > 0, 1].mean()),
                epoch_loss=[float(v) for v in out["losses"]])
    return GateModel(out["params"], out["mu"], out["sigma"], band_lo=lo, band_hi=hi, info=info)


# ---------------------------------------------------------------- stop head

STOP_RULES = ("hop", "rank", "ratio")


def stop_scores(calc: Calculator, model: GateModel, rows: np.ndarray, pool: int) -> tuple[np.ndarray, dict]:
    """Per expansion source row: the trained stop head's logit (evaluated by
    the device code the search runs, calculator_rover_gate_eval) and the
    single-feature scores of the method without the network -- hop count,
    pool rank of the source, source distance / worst pool distance (higher
    = stop sooner).  Returns (source rows, {name: score})."""
    src = rows[(rows["flags"] & SOURCE) != 0]
    raw = np.stack([src["quantized"], src["rank"], src["worst"], src["hop"].astype(np.float32) / np.float32(pool),
                    src["qnorm"]], 1).astype(np.float32)
    model.load(calc)
    logits = calc.gate_eval(raw)
    scores = {"network": logits[:, 1].astype(np.float64), "hop": src["hop"].astype(np.float64),
              "rank": src["rank"].astype(np.float64),
              "ratio": (src["quantized"] / np.maximum(src["worst"], 1e-30)).astype(np.float64)}
    return src, scores


def stop_savings(rows: np.ndarray, ids: np.ndarray, counts: np.ndarray, scores: dict, top_k: int = 10,
                 budgets=(0.002, 0.005, 0.01, 0.02), thresholds: int = 200) -> dict:
    """For each stop score and loss budget: the largest share of a trace's
    expansions that a threshold on the score saves (and that threshold) (each query stops before its first source whose
    score passes the threshold) while losing at most `budget` of the final
    top-k results (a result is lost when it was first scored at or after the
    stopping hop -- the stop label of `labels`).  `rows` are the full trace
    rows of the queries `ids` / `counts` (the search's final results); the
    scores are aligned with the source rows in trace order."""
    nq = ids.shape[0]
    src_mask = (rows["flags"] & SOURCE) != 0
    src = rows[src_mask]
    q = src["query"].astype(np.int64)
    hop = src["hop"].astype(np.int64)
    order = np.lexsort((hop, q))
    q, hop = q[order], hop[order]
    total = np.bincount(q, minlength=nq)
    starts = np.concatenate([[0], np.cumsum(total)[:-1]])
    # hop at which each final result was first scored (seeds: -1)
    k = np.minimum(counts, top_k)
    span = np.int64(1) << 32
    res = np.concatenate([np.int64(i) * span + ids[i, :k[i]].astype(np.int64) for i in range(nq)]) if nq else \
        np.zeros(0, np.int64)
    cand = rows[~src_mask]
    key = cand["query"].astype(np.int64) * span + cand["id"].astype(np.int64)
    hit = np.isin(key, res)
    found_hop = np.where((cand["flags"][hit] & SEED) != 0, -1, cand["hop"][hit]).astype(np.int64)
    found_q = cand["query"][hit].astype(np.int64)
    out = {}
    n = len(q)
    has = total > 0
    for name, s in scores.items():
        s = np.asarray(s, np.float64)[order]
        best = {str(b): {"saved": 0.0, "threshold": float("inf")} for b in budgets}
        for t in np.unique(np.quantile(s, np.linspace(0.0, 1.0, thresholds))) if n else []:
            idx = np.where(s > t, np.arange(n), n)
            first = np.full(nq, n, np.int64)
            if n:
                first[has] = np.minimum.reduceat(idx, starts[has])
            stops = first < n
            stop_hop = np.where(stops, hop[np.minimum(first, n - 1)], np.iinfo(np.int64).max)
            saved = float(np.where(stops, total - (first - starts), 0).sum()) / max(1, int(total.sum()))
            lost = float((found_hop >= stop_hop[found_q]).sum()) / max(1, nq * top_k)
            for b in budgets:
                if lost <= b and saved > best[str(b)]["saved"]:
                    best[str(b)] = {"saved": saved, "threshold": float(t)}
        out[name] = best
    return out
