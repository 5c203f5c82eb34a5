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
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--form", default="gated", choices=("plain", "packed", "batched", "gated"))
    ap.add_argument("--workload", default="pq_1m_d128")
    ap.add_argument("--queries", type=int, default=2000)
    ap.add_argument("--L", type=int, default=32)
    ap.add_argument("--ep", type=int, default=4096)
    ap.add_argument("--W", type=int, default=2)
    ap.add_argument("--repeat", type=int, default=1)
    ap.add_argument("--cache-dir", default=os.environ.get("ROVER_BENCH_CACHE", "/tmp/rover_bench_cache"))
    args = ap.parse_args(argv)

    from . import workloads
    from .calculator import GATE_PARAMS, MODE_BATCHED, MODE_EXACT, MODE_GATED, Calculator
    w = workloads.build_pq(args.workload, cache_dir=args.cache_dir, verbose=False)
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
    calc.pq_search(q, args.L, **kw)
    warm = calc.launch_count() - l0
    calc.kernel_timing(True)
    for _ in range(args.repeat):
        calc.pq_search(q, args.L, **kw)
    times = {k: v[1] / args.repeat for k, v in calc.kernel_times().items() if v[0] > 0}
    calc.kernel_timing(False)
    print(json.dumps(dict(form=args.form, workload=args.workload, queries=len(q), L=args.L, entry_points=args.ep,
                          beam_width=args.W if args.form in ("batched", "gated") else None,
                          warm_launches=warm, kernel_ms=times)), flush=True)
    calc.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
