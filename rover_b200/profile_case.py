"""One search of a chosen form on a benchmark workload, for profilers.

    python -m rover_b200.profile_case --form gated --queries 2000

Builds (or loads from --cache-dir) the workload, loads the index, runs the
search once untimed (decoded rows, seed reconstructions and scratch are
built then), then runs it --repeat more times and prints one JSON line with
the per-kernel CUDA-event times of those runs.  A profiler attached to the
process captures the kernels of the repeated runs with a launch skip equal
to the first run's launch count, which the line reports as ``warm_launches``.

Forms: ``plain`` (exact mode, decoded rows), ``packed`` (exact mode, packed
residual rows), ``batched`` (W-wide steps, full correction) and ``gated``
(the batched kernel with a loaded gate whose thresholds correct every
shortlisted seed and never stop -- the configuration bench.py's calibration
keeps on the 1M x 128 workload).

``--form sq`` runs the SQ drop-in's search (the 20,000 x 128 SQ8 workload,
SQMD, L = 64, expand 32, exact residual correction, the top 20 returned) on
--queries queries with --ep entry points.

``--form score --kind K`` runs one of the batched distance kernels of
calculator_rover_score instead (K: 0 ADC, 1 packed residual, 2 SQ8 code
distance, 3 SQ exact residual, 4 decoded-row rescore) on --queries queries x
--ids uniformly random ids over the index; ``--form refine`` the FP64 final
refine of 128 candidates per query.  SQ kinds encode the same base vectors
with the global 8-bit SQ codec.  With ``--adc-n N`` (kind 0) the index is a
synthetic one of N random M=16 codes, so that the gathered codes exceed L2.
"""

from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--form", default="gated",
                    choices=("plain", "packed", "batched", "gated", "score", "refine", "sq"))
    ap.add_argument("--kind", type=int, default=4)
    ap.add_argument("--ids", type=int, default=8192)
    ap.add_argument("--adc-n", type=int, default=0)
    ap.add_argument("--workload", default="pq_1m_d128")
    ap.add_argument("--queries", type=int, default=2000)
    ap.add_argument("--L", type=int, default=32)
    ap.add_argument("--ep", type=int, default=4096)
    ap.add_argument("--W", type=int, default=2)
    ap.add_argument("--repeat", type=int, default=1)
    ap.add_argument("--cache-dir", default=os.environ.get("ROVER_BENCH_CACHE", "/tmp/rover_bench_cache"))
    ap.add_argument("--layout", default="original", choices=("original", "gorder"),
                    help="gorder: the index in the neighbourhood-aware id order (rover_b200.layout)")
    args = ap.parse_args(argv)

    from . import workloads
    from .calculator import GATE_PARAMS, MODE_BATCHED, MODE_EXACT, MODE_GATED, Calculator
    if args.form in ("score", "refine"):
        return distance_case(args)
    if args.form == "sq":
        return sq_case(args)
    w = workloads.build_pq(args.workload, cache_dir=args.cache_dir, verbose=False)
    if args.layout == "gorder":
        from .layout import gorder_workload
        w, _ = gorder_workload(w)
    calc = Calculator()
    calc.pq_load(w.graph, w.entry, w.bundle)
    q = np.ascontiguousarray(w.queries[:args.queries])
    kw = dict(entry_points=args.ep, expand_count=int(w.graph.shape[1]), correction=1, refine_budget=20,
              top_k=10, stats=False)
    if args.form == "plain":
        kw.update(mode=MODE_EXACT, layout=2)
    elif args.form == "packed":
        kw.update(mode=MODE_EXACT, layout=1)
    elif args.form == "batched":
        kw.update(mode=MODE_BATCHED, beam_width=args.W)
    else:
        params = np.random.default_rng(0).normal(0, 0.1, GATE_PARAMS).astype(np.float32)
        calc.gate_load(params, np.zeros(5, np.float32), np.ones(5, np.float32), band_lo=np.inf, band_hi=np.inf,
                       refine_logit=-np.inf, stop_logit=np.inf)
        kw.update(mode=MODE_GATED, beam_width=args.W)
    l0 = calc.launch_count()
    first = calc.pq_search(q, args.L, **dict(kw, stats=True))
    warm = calc.launch_count() - l0
    st = first["stats"].astype(np.float64).mean(axis=0)
    calc.kernel_timing(True)
    for _ in range(args.repeat):
        r = calc.pq_search(q, args.L, **kw)
    times = {k: v[1] / args.repeat for k, v in calc.kernel_times().items() if v[0] > 0}
    calc.kernel_timing(False)
    recall = workloads.recall_at_k(r["ids"], r["counts"], w.gt[:len(q)], 10) if args.repeat > 0 else None
    print(json.dumps(dict(form=args.form, workload=args.workload, layout=args.layout, queries=len(q), L=args.L,
                          entry_points=args.ep, beam_width=args.W if args.form in ("batched", "gated") else None,
                          warm_launches=warm, kernel_ms=times, recall_at_10=recall,
                          scored=st[0], corrected=st[1], expanded=st[2])), flush=True)
    calc.close()
    return 0


def sq_case(args) -> int:
    """One warm-up SQMD search and --repeat timed ones on the SQ workload."""
    from . import workloads
    from .calculator import Calculator
    w = workloads.build_sq("sq_20k_d128")
    calc = Calculator()
    calc.sq_load(w.graph, w.entry, w.bundle)
    q = np.ascontiguousarray(w.queries[:args.queries])
    kw = dict(sq_mode=1, num_out=20, entry_points=args.ep, expand_count=32, correction=1)
    l0 = calc.launch_count()
    r = calc.sq_search(q, 64, 20, **kw)
    warm = calc.launch_count() - l0
    calc.kernel_timing(True)
    for _ in range(args.repeat):
        r = calc.sq_search(q, 64, 20, **kw)
    times = {k: v[1] / args.repeat for k, v in calc.kernel_times().items() if v[0] > 0}
    calc.kernel_timing(False)
    st = r["stats"].astype(np.float64).mean(axis=0)
    print(json.dumps(dict(form="sq", workload="sq_20k_d128", queries=len(q), L=64, entry_points=args.ep,
                          warm_launches=warm, kernel_ms=times, scored=st[0], turns=st[2])), flush=True)
    calc.close()
    return 0


def distance_case(args) -> int:
    """One warm-up call and --repeat timed calls of a distance kernel."""
    from . import bundle as B
    from . import datasets as D
    from . import workloads
    from .calculator import Calculator
    rng = np.random.default_rng(7)
    calc = Calculator()
    if args.form == "score" and args.kind == 0 and args.adc_n:
        n, dim, m = args.adc_n, 128, 16
        book = rng.normal(size=(m, 256, dim // m)).astype(np.float32)
        codes = rng.integers(0, 256, size=(n, m), dtype=np.uint8)
        bundle = B.PqBundle(B.PqMeta(b"\x07" * 16, n, dim, m, 256, dim // m, m), book, codes)
        calc.pq_load(None, -1, bundle)
        q = rng.normal(size=(args.queries, dim)).astype(np.float32)
        label = f"synthetic {n:,} x M=16 codes"
    else:
        w = workloads.build_pq(args.workload, cache_dir=args.cache_dir, verbose=False)
        n = w.bundle.meta.num_vectors
        q = np.ascontiguousarray(w.queries[:args.queries])
        label = args.workload
        if args.form == "score" and args.kind in (2, 3):
            cfg = workloads.CONFIGS[args.workload]
            base = D.gmm(cfg["n"], cfg["dim"], cfg["comps"], cfg["seed"], clip_nonneg=cfg["clip"],
                         normalize=cfg["normalize"])
            s, z, l1, res, qp = D.sq_encode(base, 8, 8)
            del base
            calc.sq_load(w.graph, w.entry, B.SqBundle(n, cfg["dim"], 8, float(s), float(z), l1, 8, res, qp))
        else:
            calc.pq_load(w.graph, w.entry, w.bundle)
    if args.form == "score":
        lists = list(rng.integers(0, n, size=(len(q), args.ids), dtype=np.int64).astype(np.int32))
        run = lambda: calc.score(args.kind, q, lists)
    else:
        cand = ((rng.integers(0, n, size=(len(q), 1)) + np.arange(128)[None, :] * 7919) % n).astype(np.int32)
        run = lambda: calc.refine(1, q, cand, np.full(len(q), 128, np.int32), 10)
    l0 = calc.launch_count()
    run()
    warm = calc.launch_count() - l0
    calc.kernel_timing(True)
    for _ in range(args.repeat):
        run()
    times = {k: v[1] / args.repeat for k, v in calc.kernel_times().items() if v[0] > 0}
    calc.kernel_timing(False)
    print(json.dumps(dict(form=args.form, kind=args.kind if args.form == "score" else None, index=label,
                          queries=len(q), ids_per_query=args.ids if args.form == "score" else 128,
                          warm_launches=warm, kernel_ms=times)), flush=True)
    calc.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
