"""Synthetic stand-ins for the Rover benchmark configurations.

The reference measures on SIFT-like datasets that are not part of this
project; seeded Gaussian mixtures with the configured sizes, dimensions and
value distributions stand in for them (rover_b200.datasets).  A workload is
built once per process (and optionally cached on local disk as .npy files),
then loaded into the library.

``pq_1m_d128``: base n=1,000,000 d=128 from a 1,024-component mixture
(centres N(0, 4I), sigma 0.5) clipped to >= 0; 10,000 queries from the same
mixture; a degree-48 graph = 64-NN pruned by the alpha=1.2 occlusion rule to
40 neighbours plus up to 8 long-range edges to representatives of the nearest
k-means clusters (rover_b200.datasets.navigable_graph: a pure k-NN graph of
this mixture splits into one component per cluster); entry = medoid; PQ M=16 x 256 (k-means, 25 iterations, 100,000 uniform-stride
training samples); 8-bit residuals; exact top-100 ground truth.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
import time
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from . import bundle as B
from . import datasets as D


@dataclass
class PqWorkload:
    name: str
    base_shape: tuple
    queries: np.ndarray
    gt: np.ndarray            # [nq][gt_k] exact neighbours
    graph: np.ndarray         # [n][degree]
    entry: int
    bundle: B.PqBundle
    build_seconds: float = 0.0


CONFIGS = {
    "pq_1m_d128": dict(n=1_000_000, dim=128, comps=1024, clip=True, normalize=False, nq=10_000,
                       cand=64, degree=48, alpha=1.2, m=16, ks=256, iters=25, rbits=8, seed=2024),
    "pq_100k_d128": dict(n=100_000, dim=128, comps=256, clip=True, normalize=False, nq=2_000,
                         cand=64, degree=48, alpha=1.2, m=16, ks=256, iters=10, rbits=8, seed=2024),
    "pq_1m_d96": dict(n=1_000_000, dim=96, comps=512, clip=False, normalize=True, nq=20_000,
                      cand=48, degree=32, alpha=1.2, m=24, ks=256, iters=25, rbits=8, seed=2025),
}


# SQ: base n=20,000 d=128 from a 64-component mixture (centres N(0, 4I),
# sigma 0.5), 1,000 queries, exact 32-NN graph (ties by lower id), entry =
# medoid, 8-bit global SQ codec with 8-bit residuals (the reference's codec
# is one scale / zero for the whole index), exact top-100 ground truth.
SQ_CONFIGS = {
    "sq_20k_d128": dict(n=20_000, dim=128, comps=64, nq=1_000, degree=32, l1_bits=8, rbits=8, seed=2023),
}


@dataclass
class SqWorkload:
    name: str
    queries: np.ndarray
    gt: np.ndarray
    graph: np.ndarray
    entry: int
    bundle: B.SqBundle
    build_seconds: float = 0.0


def build_sq(name: str, device=None, gt_k: int = 100) -> SqWorkload:
    cfg = SQ_CONFIGS[name]
    t0 = time.time()
    base = D.gmm(cfg["n"], cfg["dim"], cfg["comps"], cfg["seed"])
    queries = D.gmm(cfg["nq"], cfg["dim"], cfg["comps"], cfg["seed"] + 1, centers_seed=cfg["seed"])
    gt = D.exact_knn(queries, base, gt_k, device=device)
    graph = D.knn_graph(base, cfg["degree"], device=device)
    entry = D.medoid(base, device=device)
    scale, zero, l1, res, qp = D.sq_encode(base, cfg["l1_bits"], cfg["rbits"])
    bundle = B.SqBundle(cfg["n"], cfg["dim"], cfg["l1_bits"], scale, zero, l1, cfg["rbits"], res, qp)
    return SqWorkload(name, queries, gt, graph, entry, bundle, time.time() - t0)


# The large combined configuration: base n=10,000,000 d=128 from a
# 4,096-component mixture (centres N(0, 4I), sigma 0.5) clipped to >= 0;
# 100,000 queries (recall on the first 10,000, exact top-100 ground truth);
# a degree-32 graph (48-NN within each point's and the two nearest other
# clusters, alpha=1.2 pruned to 24, plus up to 8 long-range edges:
# datasets.clustered_graph); PQ M=32 x 256 trained and encoded by the
# library's own GPU trainer (calculator_rover_pq_train over 100,000
# uniform-stride samples, 25 iterations; calculator_rover_pq_encode) with
# 8-bit residuals; and over the same vectors the 4-bit global SQ codec with
# 8-bit residuals.
LARGE_CONFIGS = {
    "pq_10m_d128": dict(n=10_000_000, dim=128, comps=4096, nq=100_000, gt_queries=10_000, cand=48, degree=32,
                        alpha=1.2, probe=3, m=32, ks=256, iters=25, rbits=8, l1_bits=4, sq_rbits=8, seed=2026),
    # the same recipe at 100K (parity tests against the compiled reference)
    "pq_c5_100k": dict(n=100_000, dim=128, comps=256, nq=2_000, gt_queries=1_000, cand=48, degree=32,
                       alpha=1.2, probe=3, m=32, ks=256, iters=10, rbits=8, l1_bits=4, sq_rbits=8, seed=2027),
}


@dataclass
class LargeWorkload:
    name: str
    queries: np.ndarray
    gt: np.ndarray            # [gt_queries][100]
    graph: np.ndarray
    entry: int
    pq: B.PqBundle
    sq: B.SqBundle
    build_seconds: float = 0.0
    labels: np.ndarray | None = None   # nearest mixture centre of each vector (layout.gorder_large)


def build_large(name: str, calc, device=None, verbose: bool = True) -> LargeWorkload:
    """The combined large configuration, built on the GPU (see LARGE_CONFIGS)."""
    cfg = LARGE_CONFIGS[name]
    t0 = time.time()
    log = (lambda *a: print(f"[workload {name} {time.time() - t0:6.1f}s]", *a, file=sys.stderr, flush=True)) \
        if verbose else (lambda *a: None)
    n, dim = cfg["n"], cfg["dim"]
    base, centers = D.gmm(n, dim, cfg["comps"], cfg["seed"], clip_nonneg=True, return_centers=True)
    queries = D.gmm(cfg["nq"], dim, cfg["comps"], cfg["seed"] + 1, centers_seed=cfg["seed"], clip_nonneg=True)
    log("vectors")
    gt = D.exact_knn(queries[:cfg["gt_queries"]], base, 100, device=device)
    log("ground truth")
    graph = D.clustered_graph(base, np.maximum(centers, 0.0), cfg["cand"], cfg["degree"], cfg["alpha"],
                              long_edges=8, probe=cfg["probe"], device=device)
    entry = D.medoid(base, device=device)
    log("graph", f"mean degree {float((graph >= 0).sum(1).mean()):.1f}")
    from .layout import nearest_centre
    labels = nearest_centre(base, centers)
    sample = base[D.uniform_positions(n, min(n, 100_000))]
    book = calc.pq_train(sample, cfg["m"], cfg["ks"], cfg["iters"])
    codes = calc.pq_encode(base, book)
    rcb = dim if cfg["rbits"] == 8 else (dim + 1) // 2
    rows = np.empty((n, rcb), dtype=np.uint8)
    qp = np.empty((n, 2), dtype=np.float32)
    for s0 in range(0, n, 1 << 20):
        sl = slice(s0, min(n, s0 + (1 << 20)))
        rows[sl], qp[sl] = D.quantize_residual_rint(base[sl] - D.pq_reconstruct(codes[sl], book), cfg["rbits"])
    md = B.PqMeta(hashlib.sha256(name.encode()).digest()[:16], n, dim, cfg["m"], cfg["ks"], dim // cfg["m"],
                  B.pq_code_bytes(cfg["m"], cfg["ks"]), train_count=len(sample), kmeans_iters=cfg["iters"],
                  seed=cfg["seed"])
    pq = B.PqBundle(md, book, codes, cfg["rbits"], B.pack_residual_blocks(rows), qp)
    del rows
    log("pq codes + residuals (GPU trainer and encoder)")
    scale, zero, l1, res, sqp = D.sq_encode(base, cfg["l1_bits"], cfg["sq_rbits"], chunk=1 << 18)
    sq = B.SqBundle(n, dim, cfg["l1_bits"], scale, zero, l1, cfg["sq_rbits"], res, sqp)
    log("sq4 codes + residuals")
    return LargeWorkload(name, queries, gt, graph, entry, pq, sq, time.time() - t0, labels)


def _key(cfg: dict) -> str:
    return hashlib.sha256(json.dumps(cfg, sort_keys=True).encode()).hexdigest()[:16]


def build_pq(name: str, cache_dir: str | Path | None = None, device=None, gt_k: int = 100,
             nq: int | None = None, verbose: bool = True) -> PqWorkload:
    cfg = dict(CONFIGS[name])
    if nq is not None:
        cfg["nq"] = nq
    t0 = time.time()
    cache = None
    if cache_dir:
        cache = Path(cache_dir) / f"{name}-{_key(cfg)}"
        if (cache / "done").exists():
            return _load_cache(name, cache, cfg, time.time() - t0)
    log = (lambda *a: print(f"[workload {name} {time.time() - t0:6.1f}s]", *a, file=sys.stderr, flush=True)) \
        if verbose else (lambda *a: None)
    base = D.gmm(cfg["n"], cfg["dim"], cfg["comps"], cfg["seed"], clip_nonneg=cfg["clip"],
                 normalize=cfg["normalize"])
    queries = D.gmm(cfg["nq"], cfg["dim"], cfg["comps"], cfg["seed"] + 1, centers_seed=cfg["seed"],
                    clip_nonneg=cfg["clip"], normalize=cfg["normalize"])
    log("vectors")
    gt = D.exact_knn(queries, base, gt_k, device=device)
    log("ground truth")
    graph = D.navigable_graph(base, cfg["cand"], cfg["degree"], cfg["alpha"], long_edges=8,
                              clusters=cfg["comps"], device=device)
    entry = D.medoid(base, device=device)
    log("graph", f"mean degree {float((graph >= 0).sum(1).mean()):.1f}")
    book, codes, rows, qp = D.pq_prepare(base, cfg["m"], cfg["ks"], cfg["iters"], cfg["rbits"], device=device)
    log("pq codes + residuals")
    md = B.PqMeta(hashlib.sha256(name.encode()).digest()[:16], cfg["n"], cfg["dim"], cfg["m"], cfg["ks"],
                  cfg["dim"] // cfg["m"], B.pq_code_bytes(cfg["m"], cfg["ks"]),
                  train_count=min(cfg["n"], 100000), kmeans_iters=cfg["iters"], seed=cfg["seed"])
    bundle = B.PqBundle(md, book, codes, cfg["rbits"], B.pack_residual_blocks(rows), qp)
    w = PqWorkload(name, base.shape, queries, gt, graph, entry, bundle, time.time() - t0)
    if cache:
        cache.mkdir(parents=True, exist_ok=True)
        for k, v in dict(queries=queries, gt=gt, graph=graph, book=book, codes=codes,
                         blocks=bundle.residual_blocks, qparams=qp).items():
            np.save(cache / f"{k}.npy", v)
        (cache / "meta.json").write_text(json.dumps(dict(entry=entry, cfg=cfg)))
        (cache / "done").write_text("1")
    return w


def _load_cache(name, cache: Path, cfg, seconds) -> PqWorkload:
    meta = json.loads((cache / "meta.json").read_text())
    ld = lambda k: np.load(cache / f"{k}.npy")
    book, codes = ld("book"), ld("codes")
    md = B.PqMeta(hashlib.sha256(name.encode()).digest()[:16], cfg["n"], cfg["dim"], cfg["m"], cfg["ks"],
                  cfg["dim"] // cfg["m"], B.pq_code_bytes(cfg["m"], cfg["ks"]),
                  train_count=min(cfg["n"], 100000), kmeans_iters=cfg["iters"], seed=cfg["seed"])
    bundle = B.PqBundle(md, book, codes, cfg["rbits"], ld("blocks"), ld("qparams"))
    return PqWorkload(name, (cfg["n"], cfg["dim"]), ld("queries"), ld("gt"), ld("graph"), meta["entry"], bundle,
                      seconds)


def training_queries(name: str, n: int, offset: int = 7) -> np.ndarray:
    """Held-out queries from the workload's mixture (same centres, another
    sample seed) for training the learned gate."""
    cfg = CONFIGS[name]
    return D.gmm(n, cfg["dim"], cfg["comps"], cfg["seed"] + offset, centers_seed=cfg["seed"],
                 clip_nonneg=cfg["clip"], normalize=cfg["normalize"])


def held_out_set(name: str, n: int, offset: int, cache_dir: str | Path | None = None, gt_k: int = 100,
                 device=None) -> tuple[np.ndarray, np.ndarray]:
    """Held-out queries (training_queries with this seed offset) and their
    exact top-gt_k neighbours among the workload's base vectors: the set an
    operating point is calibrated on, kept apart from the timed queries."""
    cfg = CONFIGS[name]
    path = None
    if cache_dir:
        path = Path(cache_dir) / f"{name}-{_key(cfg)}" / f"heldout-{offset}-{n}-{gt_k}.npz"
        if path.exists():
            z = np.load(path)
            return z["queries"], z["gt"]
    base = D.gmm(cfg["n"], cfg["dim"], cfg["comps"], cfg["seed"], clip_nonneg=cfg["clip"],
                 normalize=cfg["normalize"])
    queries = training_queries(name, n, offset)
    gt = D.exact_knn(queries, base, gt_k, device=device)
    if path:
        path.parent.mkdir(parents=True, exist_ok=True)
        np.savez(path, queries=queries, gt=gt)
    return queries, gt


def recall_at_k(ids: np.ndarray, counts: np.ndarray, gt: np.ndarray, k: int) -> float:
    """demo_recall_hits_at_k (retrieval_rpc_demo_support.c:1709) averaged:
    hits among the first k results that appear in the first k truth ids."""
    hits = 0
    for i in range(ids.shape[0]):
        c = min(int(counts[i]), k)
        hits += len(np.intersect1d(ids[i, :c], gt[i, :k]))
    return hits / (ids.shape[0] * k)
