"""The reference's own host over this library: the drop-in check of the C-ABI.

oracle/_ref/rover_ref_gpu is the unmodified reference `Rover` host
(src/app/main.c, config.c and the retrieval host objects, compiled from the
reference sources by oracle/Makefile) linked against
rover_b200/lib/libcalculator.so instead of the DSP skeleton.  Its searches
go through the lane-protocol sessions this library serves on the GPU
(calculator_retrieval_pure_pq_sqmd_run for --method pq,
calculator_retrieval_expand_sqmd_run for --method sq) and the DMA index
loaders.  On every golden bundle and option set recorded from the reference
CLI over its own DSP skeleton (tests/golden/make_cli_golden.py), its
results.jsonl must be byte-identical, its recall line equal and, for pure
PQ, the metrics row's result columns (search-pool fingerprint, corrected and
refined candidate totals) equal.
"""
from __future__ import annotations

import csv
import io
import json
import os
import re
import subprocess
from pathlib import Path

import pytest

from conftest import GOLDEN, PQ_FIXTURES, SQ_FIXTURES, same_results

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
HOST = ROOT / "oracle" / "_ref" / "rover_ref_gpu"


def _cases():
    out = []
    for name in PQ_FIXTURES + SQ_FIXTURES:
        for tag in json.loads((GOLDEN / name / "cli_cases.json").read_text()):
            out.append((name, tag))
    return out


def _recalls(text):
    m = re.search(r"R@1=\s*([\d.]+) R@10=\s*([\d.]+) R@100=\s*([\d.]+)", text)
    assert m, text
    return tuple(float(x) for x in m.groups())


@pytest.mark.parametrize("name,tag", _cases())
def test_reference_host_over_this_library(name, tag, tmp_path):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    if not HOST.exists():
        pytest.skip("oracle/_ref/rover_ref_gpu was not built (reference sources absent at build time)")
    d = GOLDEN / name
    args = [a.replace("{dir}", str(d)) for a in json.loads((d / "cli_cases.json").read_text())[tag]]
    res, met = tmp_path / "results.jsonl", tmp_path / "metrics.csv"
    env = dict(os.environ, ROVER_SESSION_IDLE_MS="30000")
    p = subprocess.run([str(HOST), "search", *args, "--output", str(res), "--metrics", str(met)],
                       capture_output=True, text=True, timeout=300, cwd=tmp_path, env=env)
    assert p.returncode == 0, (p.stdout + p.stderr)[-3000:]
    assert same_results(res.read_bytes(), (d / f"cli_{tag}.jsonl").read_bytes(), tag)
    assert _recalls(p.stdout) == _recalls((d / f"cli_{tag}.out").read_text())
    ref_csv = d / f"cli_{tag}.csv"
    if ref_csv.exists():
        ours = next(csv.DictReader(io.StringIO(met.read_text())))
        ref = next(csv.DictReader(io.StringIO(ref_csv.read_text())))
        for col in ("recall_at_1", "recall_at_10", "recall_at_100", "search_pool_fingerprint", "refine_candidates",
                    "corrected_candidates", "work_items", "source_jobs", "source_retired"):
            assert ours[col] == ref[col], col
