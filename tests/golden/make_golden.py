#!/usr/bin/env python3
"""Generate the golden fixtures under tests/golden/ (run in a checkout where
the reference is available; the outputs are committed, this script is how
they were made).

For each fixture it
  1. draws a seeded Gaussian-mixture base set and queries,
  2. writes the index members with the REFERENCE's own writers, imported from
     the reference checkout: tools/build_pure_pq_index.py (engine numpy),
     tools/build_pure_pq_residual.py, tools/encode_l1_residual.py and
     tools/index_bundle.py's write_graph / record,
  3. runs the reference's compiled search code (oracle/_ref, built from the
     reference sources by oracle/Makefile) on that bundle and stores its
     outputs -- LUTs, ADC and residual distances, search pools, refined top-k,
     per-query statistics -- in golden.npz,
  4. stores the reference's independent NumPy ADC known-answer values
     (build_pure_pq_index.reference_adc) next to them.

Usage: python tests/golden/make_golden.py --reference REFERENCE_CHECKOUT (or $ROVER_REFERENCE)
"""
from __future__ import annotations

import argparse
import os
import hashlib
import json
import shutil
import sys
import tempfile
from argparse import Namespace
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from rover_b200 import bundle as B  # noqa: E402
from rover_b200 import datasets as D  # noqa: E402
from oracle import bindings  # noqa: E402

GOLDEN = Path(__file__).resolve().parent

PQ_FIXTURES = [
    # name, n, dim, comps, m, code_bits, residual_bits, cand, degree, alpha, nq, seed
    ("pq8_d64", 2000, 64, 16, 8, 8, 8, 24, 16, 1.2, 24, 11),
    ("pq4_d24", 1500, 24, 12, 12, 4, 4, 16, 10, 1.2, 24, 12),
]
SQ_FIXTURES = [
    # name, n, dim, comps, sq_bits, residual_bits, degree, prune, nq, seed
    ("sq8_d32", 2000, 32, 16, 8, 8, 12, True, 24, 21),
    ("sq4_d24", 1500, 24, 12, 4, 4, 10, False, 24, 22),
]


def _sha(path):
    return hashlib.sha256(Path(path).read_bytes()).hexdigest()


def make_pq(ref_tools, ref, name, n, dim, comps, m, code_bits, rbits, cand, degree, alpha, nq, seed):
    import build_pure_pq_index as pqb
    import build_pure_pq_residual as pqr
    import index_bundle as ib
    out = GOLDEN / name
    if out.exists():
        shutil.rmtree(out)
    out.mkdir(parents=True)
    base = D.gmm(n, dim, comps, seed)
    queries = D.gmm(nq, dim, comps, seed + 1000, centers_seed=seed)
    with tempfile.TemporaryDirectory() as tmp:
        base_path = Path(tmp) / "base.fvecs"
        B.write_fvecs(base_path, base)
        pqb.build(Namespace(base=base_path, out_prefix=out / "index", num_vectors=n, dim=dim, m=m,
                            code_bits=code_bits, ks=None, train_max=100000, kmeans_iters=8,
                            chunk_vectors=512, memory_budget_mb=64, layout_id="original", order_map=None,
                            engine="numpy", threads=1, seed=seed, force=True))
        pqr.build(Namespace(prefix=out / "index", base=base_path, num_vectors=n, residual_bits=rbits,
                            chunk_vectors=512, order_map=None, force=True))
        raw_sha = ib.sha(base_path)
        graph = D.pruned_graph(base, cand, degree, alpha, device="cpu")
        entry = D.medoid(base, device="cpu")
        ib.write_graph(out / "graph.rover", graph, dim)
        B.write_fvecs(out / "queries.fvecs", queries)
        files = {"graph": ib.record(out / "graph.rover", out)}
        suffix = f".pqres{rbits}"
        for key, ext in (("pq_book", ".pqbook"), ("pq_codes", ".pqcodes"), ("pq_manifest", ".pq.json"),
                         ("pq_residual", suffix), ("pq_qparams", suffix + ".qparams"),
                         ("pq_residual_manifest", suffix + ".json")):
            files[key] = ib.record(Path(str(out / "index") + ext), out)
        data = dict(schema=ib.SCHEMA, n=n, dim=dim, graph_degree=degree, method="pq", residual_bits=rbits,
                    third_residual=False, reordered=False, layout="original",
                    layout_hash=hashlib.sha256(b"original").hexdigest(), graph_format="rover",
                    graph_entry=entry, files=files, raw_sha256=raw_sha, residual_layout="a",
                    pq_bits=code_bits, pq_m=m, train_samples=100000, train_iters=8, seed=seed)
        ib.atomic_json(out / "index.json", data)
        B.write_fvecs(Path(tmp) / "q.fvecs", queries)
        sample = [int(i) for i in np.random.default_rng(seed).choice(n, 32, replace=False)]
        known = [pqb.reference_adc(out / "index", Path(tmp) / "q.fvecs", qi, sample) for qi in range(4)]
    # golden outputs from the compiled reference
    h = ref.pq_open(out / "index", rbits)
    md = B.read_pq_bundle(out / "index", rbits).meta
    g = {}
    ids = np.random.default_rng(seed + 7).choice(n, 64, replace=False).astype(np.int32)
    g["sample_ids"] = ids
    g["lut"] = np.stack([ref.pq_lut(h, queries[q], md.m, md.ks) for q in range(4)])
    g["adc"] = np.stack([ref.pq_adc(h, g["lut"][q], ids) for q in range(4)])
    g["residual"] = np.stack([ref.pq_residual_eval(h, queries[q], ids) for q in range(4)])
    g["known_adc_ids"] = np.asarray(sample, dtype=np.int32)
    g["known_adc"] = np.asarray([[r["distance"] for r in k] for k in known], dtype=np.float64)
    pools = np.asarray([[12, 16, 24, 32, 40, 48][i % 6] for i in range(nq)]).astype(np.int32)
    g["pool_sizes"] = pools
    for tag, corr, ep, exp in (("on", 1, 1, degree), ("off", 0, 1, degree), ("on_ep8", 1, 8, degree),
                               ("on_exp6", 1, 4, 6)):
        r = ref.pq_search(h, graph, entry, queries, pools, ep, exp, correction=corr,
                          refine_budget=20 if corr else 0, top_k=10)
        g[f"search_{tag}_pool_ids"] = r["pool_ids"]
        g[f"search_{tag}_pool_dists"] = r["pool_dists"]
        g[f"search_{tag}_pool_counts"] = r["pool_counts"]
        g[f"search_{tag}_ids"] = r["ids"]
        g[f"search_{tag}_dists"] = r["dists"]
        g[f"search_{tag}_counts"] = r["counts"]
        g[f"search_{tag}_stats"] = r["stats"]
        g[f"search_{tag}_params"] = np.asarray([corr, ep, exp], dtype=np.int32)
    ref.pq_close(h)
    np.savez_compressed(out / "golden.npz", **g)
    manifest = dict(kind="pq", n=n, dim=dim, m=m, code_bits=code_bits, residual_bits=rbits, degree=degree,
                    graph_entry=entry, seed=seed, nq=nq,
                    files={p.name: _sha(p) for p in sorted(out.iterdir()) if p.name != "manifest.json"})
    (out / "manifest.json").write_text(json.dumps(manifest, indent=2) + "\n")


def make_sq(ref_tools, ref, name, n, dim, comps, sq_bits, rbits, degree, prune, nq, seed):
    import encode_l1_residual as enc
    import index_bundle as ib
    out = GOLDEN / name
    if out.exists():
        shutil.rmtree(out)
    out.mkdir(parents=True)
    base = D.gmm(n, dim, comps, seed)
    queries = D.gmm(nq, dim, comps, seed + 1000, centers_seed=seed)
    with tempfile.TemporaryDirectory() as tmp:
        base_path = Path(tmp) / "base.fvecs"
        B.write_fvecs(base_path, base)
        enc.encode(base_path, out / "l1.bin", out / "residual.bin", out / "qparams.bin", sq_bits, rbits, 512)
        raw_sha = ib.sha(base_path)
    graph = D.pruned_graph(base, degree + 8, degree, 1.2, device="cpu") if prune else \
        D.knn_graph(base, degree, device="cpu")
    entry = D.medoid(base, device="cpu")
    ib.write_graph(out / "graph.rover", graph, dim)
    B.write_fvecs(out / "queries.fvecs", queries)
    files = {"graph": ib.record(out / "graph.rover", out)}
    for key in ("l1", "residual", "qparams"):
        files[key] = ib.record(out / f"{key}.bin", out)
    data = dict(schema=ib.SCHEMA, n=n, dim=dim, graph_degree=degree, method="sq", residual_bits=rbits,
                third_residual=False, reordered=False, layout="original",
                layout_hash=hashlib.sha256(b"original").hexdigest(), graph_format="rover", graph_entry=entry,
                files=files, raw_sha256=raw_sha, residual_layout="a", sq_bits=sq_bits)
    ib.atomic_json(out / "index.json", data)
    b = B.read_sq_bundle(out / "l1.bin", out / "residual.bin", out / "qparams.bin")
    hs = ref.sq_open(b)
    g = {}
    ids = np.random.default_rng(seed + 7).choice(n, 64, replace=False).astype(np.int32)
    g["sample_ids"] = ids
    g["query_codes"] = np.stack([ref.sq_quantize(hs, queries[q]) for q in range(nq)])
    g["coarse"] = np.stack([ref.sq_coarse(hs, queries[q], ids) for q in range(4)])
    g["exact"] = np.stack([ref.sq_exact(hs, queries[q], ids) for q in range(4)])
    pools = np.asarray([[10, 16, 24, 32, 48, 64][i % 6] for i in range(nq)]).astype(np.int32)
    g["pool_sizes"] = pools
    for tag, corr, ep, exp in (("on", 1, 1, degree), ("off", 0, 1, degree), ("on_ep8", 1, 8, degree),
                               ("off_ep16_exp5", 0, 16, 5)):
        r = ref.sqmd_search(hs, graph, entry, queries, pools, ep, exp, correction=corr, lanes=4)
        g[f"sqmd_{tag}_ids"] = r["ids"]
        g[f"sqmd_{tag}_dists"] = r["dists"]
        g[f"sqmd_{tag}_counts"] = r["counts"]
        g[f"sqmd_{tag}_params"] = np.asarray([corr, ep, exp], dtype=np.int32)
        if corr:
            rc = np.minimum(r["counts"], 20)
            ri, rd, rn = ref.refine(0, hs, queries, r["ids"], r["dists"], rc, 10)
            g[f"sqmd_{tag}_refine_ids"] = ri
            g[f"sqmd_{tag}_refine_dists"] = rd
            g[f"sqmd_{tag}_refine_counts"] = rn
    for tag, ep, exp, num_out in (("ep1", 1, degree, 20), ("ep8", 8, degree, 20), ("ep4_exp4", 4, 4, 30)):
        r = ref.dsp_search(b, graph, entry, queries, pools, ep, exp, num_out)
        g[f"dsp_{tag}_ids"] = r["ids"]
        g[f"dsp_{tag}_dists"] = r["dists"]
        g[f"dsp_{tag}_counts"] = r["counts"]
        g[f"dsp_{tag}_params"] = np.asarray([ep, exp, num_out], dtype=np.int32)
    ref.sq_close(hs)
    np.savez_compressed(out / "golden.npz", **g)
    manifest = dict(kind="sq", n=n, dim=dim, sq_bits=sq_bits, residual_bits=rbits, degree=degree,
                    graph_entry=entry, seed=seed, nq=nq,
                    files={p.name: _sha(p) for p in sorted(out.iterdir()) if p.name != "manifest.json"})
    (out / "manifest.json").write_text(json.dumps(manifest, indent=2) + "\n")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("ROVER_REFERENCE"),
                    required="ROVER_REFERENCE" not in os.environ,
                    help="reference checkout (default: $ROVER_REFERENCE)")
    args = ap.parse_args()
    tools = Path(args.reference) / "tools"
    sys.path.insert(0, str(tools))
    bindings.build(args.reference)
    ref = bindings.Reference()
    for f in PQ_FIXTURES:
        print("fixture", f[0], flush=True)
        make_pq(tools, ref, *f)
    for f in SQ_FIXTURES:
        print("fixture", f[0], flush=True)
        make_sq(tools, ref, *f)


if __name__ == "__main__":
    main()
