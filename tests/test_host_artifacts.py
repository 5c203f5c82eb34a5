"""The C host's correction artifacts on the CPU (rover_b200/host/artifacts.c):
the ERROR4 file of the final refine's mode 2 and the SQ4 split-distance bias,
read from the golden fixtures (written by the reference's own tools) and
checked the way the reference host checks them (retrieval_final_refine.c:
118-166, retrieval_rpc_demo_support.c:237-297): what loads must equal the
file's payload; a changed byte, header field, base member, codebook or id
map must be refused.  The command line's option rules are checked too."""
from __future__ import annotations

import ctypes as C
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from conftest import GOLDEN, PQ_FIXTURES, SQ_FIXTURES

ROOT = Path(__file__).resolve().parents[1]
HOST = ROOT / "rover_b200" / "lib" / "librover_host.so"
ROVER = ROOT / "rover_b200" / "bin" / "Rover"


class Error4(C.Structure):
    _fields_ = [("num_vectors", C.c_int32), ("dim", C.c_int32), ("qparams", C.c_void_p), ("blocks", C.c_void_p),
                ("blocks_bytes", C.c_int64), ("file", C.c_void_p)]


@pytest.fixture(scope="module")
def host():
    if not HOST.exists() or not ROVER.exists():
        from rover_b200 import build
        build.build_host()
    lib = C.CDLL(str(HOST))
    lib.rover_bundle_open_dir.argtypes = [C.c_char_p, C.c_int, C.POINTER(C.c_void_p)]
    lib.rover_bundle_close.argtypes = [C.c_void_p]
    lib.rover_host_error.restype = C.c_char_p
    lib.rover_error4_open.argtypes = [C.c_void_p, C.c_char_p, C.c_void_p, C.POINTER(C.POINTER(Error4))]
    lib.rover_error4_close.argtypes = [C.POINTER(Error4)]
    lib.rover_split_bias_open.argtypes = [C.c_void_p, C.c_char_p, C.POINTER(C.POINTER(C.c_float))]
    lib.rover_artifact_error.restype = C.c_char_p
    return lib


def _bundle(host, d, verify=1):
    b = C.c_void_p()
    assert host.rover_bundle_open_dir(str(d).encode(), verify, C.byref(b)) == 0, host.rover_host_error()
    return b


def _error4(host, b, path, order=None):
    e = C.POINTER(Error4)()
    m = None if order is None else np.ascontiguousarray(order, dtype=np.int32)
    rc = host.rover_error4_open(b, str(path).encode(), None if m is None else m.ctypes.data, C.byref(e))
    return rc, e, host.rover_artifact_error().decode()


@pytest.mark.parametrize("name", PQ_FIXTURES + SQ_FIXTURES)
def test_error4_loads_the_artifact_payload(host, name):
    from oracle.bindings import read_error4
    import json
    d = GOLDEN / name
    data = json.loads((d / "index.json").read_text())
    b = _bundle(host, d)
    try:
        rc, e, err = _error4(host, b, d / "error4.refine")
        assert rc == 0, err
        n, dim = data["n"], data["dim"]
        qp, blocks, _, _ = read_error4(d / "error4.refine", n, dim)
        got_qp = np.ctypeslib.as_array(C.cast(e.contents.qparams, C.POINTER(C.c_float)), shape=(n * 2,))
        got_blocks = np.ctypeslib.as_array(C.cast(e.contents.blocks, C.POINTER(C.c_uint8)),
                                           shape=(e.contents.blocks_bytes,))
        assert np.array_equal(got_qp.reshape(n, 2), qp) and np.array_equal(got_blocks, blocks)
        host.rover_error4_close(e)
        # an order map changes the id-map digest the artifact is bound to
        rc, _, err = _error4(host, b, d / "error4.refine", order=np.arange(n)[::-1])
        assert rc != 0 and "id-map" in err
    finally:
        host.rover_bundle_close(b)


def _corrupt(src: Path, dst: Path, offset: int, value=None, truncate=None):
    raw = bytearray(src.read_bytes())
    if truncate is not None:
        raw = raw[:truncate]
    else:
        raw[offset] = (raw[offset] ^ 0xFF) if value is None else value
    dst.write_bytes(bytes(raw))
    return dst


def test_error4_refuses_what_the_reference_refuses(host, tmp_path):
    d = tmp_path / "pq8_d64"
    shutil.copytree(GOLDEN / "pq8_d64", d)
    src = d / "error4.refine"
    b = _bundle(host, d)
    try:
        for tag, kw, want in (("magic", dict(offset=0, value=ord("S")), "header"),
                              ("version", dict(offset=8, value=2), "header"),
                              ("block", dict(offset=29, value=0), "header"),
                              ("payload", dict(offset=300), "payload digest"),
                              ("base", dict(offset=90), "base members"),
                              ("book", dict(offset=186), "codebook"),
                              ("size", dict(offset=0, truncate=4000), "header")):
            bad = _corrupt(src, tmp_path / f"e4_{tag}", **kw)
            rc, _, err = _error4(host, b, bad)
            assert rc != 0 and want in err, (tag, err)
        # the SQ magic on a PQ index
        raw = bytearray(src.read_bytes())
        raw[0:8] = b"SQERR4V1"
        (tmp_path / "e4_sqmagic").write_bytes(bytes(raw))
        assert _error4(host, b, tmp_path / "e4_sqmagic")[0] != 0
    finally:
        host.rover_bundle_close(b)
    # a base member changed after the artifact was made (bundle opened without
    # its own digest checks, as the explicit --pq-* options do)
    codes = d / "index.pqcodes"
    raw = bytearray(codes.read_bytes())
    raw[-1] ^= 0x01
    codes.write_bytes(bytes(raw))
    b = _bundle(host, d, verify=0)
    try:
        rc, _, err = _error4(host, b, src)
        assert rc != 0 and "base members" in err
    finally:
        host.rover_bundle_close(b)


def test_split_bias_loads_and_refuses(host, tmp_path):
    from oracle.bindings import read_bias
    d = GOLDEN / "sq4_d24"
    b = _bundle(host, d)
    out = C.POINTER(C.c_float)()
    try:
        assert host.rover_split_bias_open(b, str(d / "correction_bias.f32").encode(), C.byref(out)) == 0, \
            host.rover_artifact_error()
        n = 1500
        assert np.array_equal(np.ctypeslib.as_array(out, shape=(n,)), read_bias(d / "correction_bias.f32", n))
        for tag, kw, want in (("magic", dict(offset=1), "header"), ("fingerprint", dict(offset=50), "header"),
                              ("payload", dict(offset=100), "hash"), ("bits", dict(offset=24, value=8), "header")):
            bad = _corrupt(d / "correction_bias.f32", tmp_path / f"bias_{tag}", **kw)
            rc = host.rover_split_bias_open(b, str(bad).encode(), C.byref(out))
            assert rc != 0 and want in host.rover_artifact_error().decode(), tag
    finally:
        host.rover_bundle_close(b)
    # 8-bit L1 codes cannot take the split distance
    b = _bundle(host, GOLDEN / "sq8_d32")
    try:
        assert host.rover_split_bias_open(b, str(d / "correction_bias.f32").encode(), C.byref(out)) != 0
        assert "4-bit" in host.rover_artifact_error().decode()
    finally:
        host.rover_bundle_close(b)


def test_cli_rules_for_the_artifacts(host):
    base = ["search", "--n", "100", "--dim", "16", "--graph-degree", "8", "--nq", "1", "--query", "q", "--graph", "g"]
    run = lambda *a: subprocess.run([str(ROVER), *a], capture_output=True, text=True, timeout=60)  # noqa: E731
    p = run(*base, "--third-residual", "on")
    assert p.returncode == 2 and "missing or unreadable third residual artifact" in p.stderr
    p = run(*base, "--third-residual", "on", "--error4", "/nonexistent/error4.refine")
    assert p.returncode == 2 and "missing or unreadable third residual artifact" in p.stderr
    p = run(*base, "--method", "sq", "--sq-bits", "8", "--split-distance", "on", "--bias", "x")
    assert p.returncode == 2 and "split distance requires SQ4 online correction" in p.stderr
    p = run(*base, "--method", "sq", "--sq-bits", "4", "--split-distance", "on")
    assert p.returncode == 2 and "split distance requires SQ4 online correction" in p.stderr
