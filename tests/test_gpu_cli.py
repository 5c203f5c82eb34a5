"""`Rover search` (bin/Rover, the C host over libcalculator.so) against the
reference's own `Rover search` run on the same bundles
(tests/golden/make_cli_golden.py): byte-identical results.jsonl, the same
recall@1/10/100 and, for pure PQ, the same search-pool fingerprint (an FNV-1a
hash over every query's pool ids and distance bits before refinement), the
same corrected-candidate and refine-candidate totals."""
from __future__ import annotations

import csv
import io
import json
import re
import subprocess
from pathlib import Path

import pytest

from conftest import GOLDEN, PQ_FIXTURES, SQ_FIXTURES, same_results

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
ROVER = ROOT / "rover_b200" / "bin" / "Rover"


def _cases():
    out = []
    for name in PQ_FIXTURES + SQ_FIXTURES:
        for tag in json.loads((GOLDEN / name / "cli_cases.json").read_text()):
            out.append((name, tag))
    return out


def _run(args, tmp_path):
    res, met = tmp_path / "results.jsonl", tmp_path / "metrics.csv"
    p = subprocess.run([str(ROVER), "search", *args, "--output", str(res), "--metrics", str(met)],
                       capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stdout + p.stderr
    return p.stdout, res.read_bytes(), met.read_text() if met.exists() else None


def _recalls(text):
    m = re.search(r"R@1=\s*([\d.]+) R@10=\s*([\d.]+) R@100=\s*([\d.]+)", text)
    assert m, text
    return tuple(float(x) for x in m.groups())


def _row(text):
    return next(csv.DictReader(io.StringIO(text)))


@pytest.mark.parametrize("name,tag", _cases())
def test_cli_matches_reference_cli(name, tag, tmp_path):
    d = GOLDEN / name
    args = [a.replace("{dir}", str(d)) for a in json.loads((d / "cli_cases.json").read_text())[tag]]
    out, results, metrics = _run(args, tmp_path)
    assert same_results(results, (d / f"cli_{tag}.jsonl").read_bytes(), tag)
    assert _recalls(out) == _recalls((d / f"cli_{tag}.out").read_text())
    if (d / f"cli_{tag}.csv").exists():
        ours, ref = _row(metrics), _row((d / f"cli_{tag}.csv").read_text())
        for col in ("recall_at_1", "recall_at_10", "recall_at_100", "search_pool_fingerprint", "refine_candidates",
                    "refine_budget", "refine_mode", "corrected_candidates", "entry_points", "pool_size", "queries",
                    "code_bits", "ks", "m", "code_bytes", "compression_x", "top_k"):
            assert ours[col] == ref[col], col


@pytest.mark.parametrize("name", [PQ_FIXTURES[0], SQ_FIXTURES[0]])
def test_index_dir_gives_the_same_results(name, tmp_path):
    """--index-dir (index.json, member checksums) instead of member paths."""
    d = GOLDEN / name
    args = [a.replace("{dir}", str(d)) for a in json.loads((d / "cli_cases.json").read_text())["refine"]]
    drop = {"--graph", "--graph-format", "--pq-prefix", "--pq-book", "--pq-codes", "--pq-residual", "--pq-qparams",
            "--l1", "--residual", "--qparams", "--layout-hash"}
    kept = []
    it = iter(args)
    for a in it:
        v = next(it) if a.startswith("--") and a != "--refine-all" else None
        if a not in drop:
            kept += [a] + ([v] if v is not None else [])
    _, results, _ = _run(kept + ["--index-dir", str(d)], tmp_path)
    assert results == (d / "cli_refine.jsonl").read_bytes()
