"""Shared fixtures.  GPU tests are marked ``gpu``; everything else runs on
the CPU (the oracle, formats, host logic and the library's exported ABI)."""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
GOLDEN = ROOT / "tests" / "golden"

PQ_FIXTURES = ["pq8_d64", "pq4_d24"]
SQ_FIXTURES = ["sq8_d32", "sq4_d24"]


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def same_results(ours: bytes, ref: bytes, tag: str) -> bool:
    """results.jsonl equality: byte for byte, except that the reference's
    DB-pair driver writes each query's line when its worker thread finishes
    (retrieval_rpc_demo_pipeline.c:2560-2620, several pairs in flight), so for
    those cases the line order is the threads' and the same set of lines is
    required instead."""
    if tag.startswith("db_pair"):
        return sorted(ours.splitlines()) == sorted(ref.splitlines())
    return ours == ref


def load_fixture(name):
    from rover_b200 import bundle as B
    d = GOLDEN / name
    data, graph, b = B.load_index_dir(d)
    golden = dict(np.load(d / "golden.npz"))
    queries = B.read_fvecs(d / "queries.fvecs")
    return data, graph, b, golden, queries


@pytest.fixture(scope="session")
def port():
    from oracle import bindings
    if not bindings.port_available():
        bindings.build()
    return bindings.Port()


@pytest.fixture(scope="session")
def calc():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from rover_b200.calculator import Calculator
    return Calculator()
