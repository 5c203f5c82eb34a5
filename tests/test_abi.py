"""The C-ABI library: it loads without a GPU and exports every function that
include/*.h declares (no compute call is made here)."""
from __future__ import annotations

import ctypes
import re
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
LIB = ROOT / "rover_b200" / "lib" / "libcalculator.so"
HEADERS = sorted((ROOT / "include").glob("*.h"))


def declared_functions():
    names = set()
    for h in HEADERS:
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        text = re.sub(r"#define[^\n]*", "", text)
        for m in re.finditer(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", text):
            name = m.group(1)
            if name.startswith(("calculator_", "rpcmem_", "fastrpc_", "remote_")):
                names.add(name)
    return sorted(names)


@pytest.fixture(scope="module")
def lib():
    if not LIB.exists():
        from rover_b200 import build
        build.build()
    return ctypes.CDLL(str(LIB))


def test_headers_declare_the_idl_surface():
    names = declared_functions()
    idl = ["calculator_open", "calculator_close", "calculator_rover_configure",
           "calculator_retrieval_async_submit", "calculator_retrieval_async_poll",
           "calculator_retrieval_async_reset", "calculator_retrieval_load", "calculator_retrieval_search",
           "calculator_retrieval_unload", "calculator_retrieval_load_dma", "calculator_retrieval_unload_dma",
           "calculator_retrieval_rnn_l2_load_dma", "calculator_retrieval_rnn_l2_batch",
           "calculator_retrieval_rnn_l2_unload_dma", "calculator_retrieval_search_db",
           "calculator_retrieval_expand_sqmd", "calculator_retrieval_expand_sqmd_run",
           "calculator_retrieval_pure_pq_load_dma", "calculator_retrieval_pure_pq_unload_dma",
           "calculator_retrieval_pure_pq_sqmd_run"]
    assert set(idl) <= set(names)


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_exports_are_c_symbols():
    out = subprocess.run(["nm", "-D", "--defined-only", str(LIB)], capture_output=True, text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    for name in declared_functions():
        assert name in exported, name


def test_configure_validates_without_a_gpu(lib):
    lib.calculator_rover_configure.argtypes = [ctypes.c_uint64, ctypes.c_int32, ctypes.c_int32]
    assert lib.calculator_rover_configure(0, 2, 4) == 14   # AEE_EBADPARM: build ABI
    assert lib.calculator_rover_configure(0, 1, 5) == 14
    assert lib.calculator_rover_configure(0, 1, 8) == 0
