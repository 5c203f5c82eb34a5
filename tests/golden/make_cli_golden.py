#!/usr/bin/env python3
"""Record the reference CLI's outputs on the golden bundles (run where the
reference is available; the outputs are committed, this script is how they
were made).

For every fixture under tests/golden/ it runs the reference's own `Rover
search` executable (oracle/_ref/rover_ref, built from the reference sources
by oracle/Makefile; its DSP side runs on the host through oracle/shim) with
a few option sets and stores, per case, the command's options
(cli_cases.json), its results.jsonl (cli_<case>.jsonl), its standard output
(cli_<case>.out) and, for PQ, its metrics CSV (cli_<case>.csv), with the
fixture directory written as {dir}.  The ground-truth file the runs evaluate
against (cli_gt.ivecs) holds, per query, the reference's own top-10 of the fixture's
first golden search padded with -1 to 100 columns.

Usage: python tests/golden/make_cli_golden.py --reference REFERENCE_CHECKOUT (or $ROVER_REFERENCE)
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from rover_b200 import bundle as B  # noqa: E402
from oracle import bindings  # noqa: E402

GOLDEN = Path(__file__).resolve().parent
FIXTURES = ["pq8_d64", "pq4_d24", "sq8_d32", "sq4_d24"]


def cases(data: dict, d: Path) -> dict:
    deg = int(data["graph_degree"])
    # the final refine's mode 2 (ERROR4 term) and the SQ4 split distance,
    # over the artifacts tests/golden/make_refine_artifacts.py wrote
    error4 = ["--third-residual", "on", "--error4", str(d / "error4.refine")]
    extra = {}
    if (d / "error4.refine").exists():
        extra["third_residual"] = ["--pool", "32", "--entry-points", "4", "--expand-count", str(min(16, deg)),
                                   "--refine", "on"] + error4
    if (d / "correction_bias.f32").exists():
        split = ["--split-distance", "on", "--bias", str(d / "correction_bias.f32")]
        extra["split_refine"] = ["--pool", "32", "--entry-points", "4", "--expand-count", str(min(16, deg)),
                                 "--refine", "on"] + split
        extra["split_first_stage"] = ["--pool", "40", "--entry-points", "8", "--expand-count", str(min(8, deg)),
                                      "--refine", "off"] + split
        extra["split_third_residual"] = ["--pool", "24", "--entry-points", "6", "--expand-count",
                                         str(min(12, deg)), "--refine", "on"] + split + error4
    if data["method"] == "pq":
        return {
            "refine": ["--pool", "32", "--entry-points", "4", "--expand-count", str(min(16, deg)), "--refine", "on"],
            "coarse_pool": ["--pool", "48", "--entry-points", "8", "--expand-count", str(min(12, deg)),
                            "--refine", "off"],
            "refine_all": ["--pool", "24", "--entry-points", "1", "--expand-count", str(deg), "--refine-all",
                           "--refine", "on", "--top-k", "5", "--seed", "7"],
            **extra,
        }
    return {
        "refine": ["--pool", "32", "--entry-points", "4", "--expand-count", str(min(16, deg)), "--refine", "on"],
        "first_stage": ["--pool", "40", "--entry-points", "8", "--expand-count", str(min(8, deg)), "--refine", "off"],
        # DB-pair search (calculator_retrieval_search_db with the host's
        # residual correction); refine off re-ranks with demo_rerank_candidates
        "db_pair_rerank": ["--search-mode", "db-pair", "--pool", "32", "--entry-points", "4",
                           "--expand-count", str(min(16, deg)), "--refine", "off"],
        "db_pair_refine": ["--search-mode", "db-pair", "--pool", "24", "--entry-points", "6",
                           "--expand-count", str(min(12, deg)), "--refine", "on"],
        **extra,
    }


def base_args(d: Path, data: dict, nq: int, gt: Path) -> list[str]:
    f = data["files"]
    args = ["--method", data["method"], "--n", str(data["n"]), "--dim", str(data["dim"]), "--nq", str(nq),
            "--graph-degree", str(data["graph_degree"]), "--graph", str(d / f["graph"]["path"]),
            "--graph-format", data.get("graph_format", "rover"), "--graph-entry", str(data["graph_entry"]),
            "--query", str(d / "queries.fvecs"), "--gt", str(gt), "--residual-bits", str(data["residual_bits"]),
            "--storage", "memory", "--correction", "online"]
    if data["method"] == "pq":
        args += ["--pq-prefix", str(d / "index"), "--pq-book", str(d / f["pq_book"]["path"]),
                 "--pq-codes", str(d / f["pq_codes"]["path"]), "--pq-residual", str(d / f["pq_residual"]["path"]),
                 "--pq-qparams", str(d / f["pq_qparams"]["path"]), "--pq-bits", str(data["pq_bits"]),
                 "--pq-m", str(data["pq_m"]), "--layout-hash", data["layout_hash"]]
    else:
        args += ["--l1", str(d / f["l1"]["path"]), "--residual", str(d / f["residual"]["path"]),
                 "--qparams", str(d / f["qparams"]["path"]), "--sq-bits", str(data["sq_bits"])]
    return args


def relative(args: list[str], d: Path) -> list[str]:
    """Fixture paths as {dir}/name so the test can substitute its own."""
    return [a.replace(str(d), "{dir}") for a in args]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("ROVER_REFERENCE"),
                    required="ROVER_REFERENCE" not in os.environ,
                    help="reference checkout (default: $ROVER_REFERENCE)")
    ap.add_argument("--tags", nargs="*", help="record only these cases (the others stay as recorded)")
    args = ap.parse_args()
    bindings.build(args.reference)
    rover_ref = ROOT / "oracle" / "_ref" / "rover_ref"
    env = dict(os.environ, LD_LIBRARY_PATH=str(ROOT / "oracle" / "_ref"))
    for name in FIXTURES:
        d = GOLDEN / name
        data = json.loads((d / "index.json").read_text())
        g = np.load(d / "golden.npz")
        nq = len(B.read_fvecs(d / "queries.fvecs"))
        key = "search_on_ids" if data["method"] == "pq" else "sqmd_on_ids"
        gt = np.full((nq, 100), -1, np.int32)
        gt[:, :10] = g[key][:, :10]
        if not args.tags:
            B.write_ivecs(d / "cli_gt.ivecs", gt)
        cases_file = d / "cli_cases.json"
        record = json.loads(cases_file.read_text()) if args.tags and cases_file.exists() else {}
        for tag, extra in cases(data, d).items():
            if args.tags and tag not in args.tags:
                continue
            with tempfile.TemporaryDirectory() as tmp:
                out, met = Path(tmp) / "results.jsonl", Path(tmp) / "metrics.csv"
                full = base_args(d, data, nq, d / "cli_gt.ivecs") + extra + ["--output", str(out), "--metrics", str(met)]
                p = subprocess.run([str(rover_ref), "search", *full], env=env, capture_output=True, text=True,
                                   timeout=300)
                if p.returncode != 0:
                    raise SystemExit(f"{name}/{tag}: reference CLI failed\n{p.stdout}\n{p.stderr}")
                (d / f"cli_{tag}.jsonl").write_bytes(out.read_bytes())
                if met.exists():      # the pure-PQ driver writes a metrics row; the SQMD driver prints only
                    (d / f"cli_{tag}.csv").write_text(met.read_text().replace(str(d), "{dir}"))
                (d / f"cli_{tag}.out").write_text(p.stdout.replace(str(d), "{dir}").replace(tmp, "{tmp}"))
                record[tag] = relative(full[:-4], d)
            print(name, tag, "ok", flush=True)
        (d / "cli_cases.json").write_text(json.dumps(record, indent=1) + "\n")


if __name__ == "__main__":
    main()
