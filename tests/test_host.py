"""The C host (librover_host.so, bin/Rover) on the CPU: SHA-256 against
hashlib, the bundle loader against the Python readers and the reference's
validation rules, the vector readers, the exported symbols, and the `Rover`
command line's option handling (no search runs here)."""
from __future__ import annotations

import ctypes as C
import hashlib
import json
import os
import re
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from conftest import GOLDEN, PQ_FIXTURES, SQ_FIXTURES, load_fixture

ROOT = Path(__file__).resolve().parents[1]
HOST = ROOT / "rover_b200" / "lib" / "librover_host.so"
ROVER = ROOT / "rover_b200" / "bin" / "Rover"


class PqDesc(C.Structure):
    _fields_ = [("graph", C.c_void_p), ("num_vectors", C.c_int32), ("graph_degree", C.c_int32),
                ("graph_entry", C.c_int32), ("dim", C.c_int32), ("codes", C.c_void_p), ("codebook", C.c_void_p),
                ("m", C.c_int32), ("ks", C.c_int32), ("subdim", C.c_int32), ("code_bytes", C.c_int32),
                ("residual_blocks", C.c_void_p), ("residual_blocks_bytes", C.c_int64),
                ("residual_bits", C.c_int32), ("residual_qparams", C.c_void_p)]


class SqDesc(C.Structure):
    _fields_ = [("graph", C.c_void_p), ("num_vectors", C.c_int32), ("graph_degree", C.c_int32),
                ("graph_entry", C.c_int32), ("dim", C.c_int32), ("l1_codes", C.c_void_p), ("l1_bits", C.c_int32),
                ("l1_scale", C.c_float), ("l1_zero", C.c_float), ("residual_rows", C.c_void_p),
                ("residual_bits", C.c_int32), ("residual_qparams", C.c_void_p)]


class Bundle(C.Structure):
    _fields_ = [("method", C.c_int32), ("n", C.c_int32), ("dim", C.c_int32), ("degree", C.c_int32),
                ("graph_entry", C.c_int32), ("residual_bits", C.c_int32), ("graph", C.c_void_p),
                ("pq", PqDesc), ("pq_codebook", C.c_void_p), ("pq_codes", C.c_void_p),
                ("pq_residual_blocks", C.c_void_p), ("pq_qparams", C.c_void_p), ("index_uuid", C.c_uint8 * 16),
                ("sq", SqDesc), ("sq_l1", C.c_void_p), ("sq_residual_rows", C.c_void_p), ("sq_qparams", C.c_void_p)]


@pytest.fixture(scope="module")
def host():
    if not HOST.exists() or not ROVER.exists():
        from rover_b200 import build
        build.build_host()
    lib = C.CDLL(str(HOST))
    lib.rover_sha256.argtypes = [C.c_void_p, C.c_size_t, C.c_char_p]
    lib.rover_sha256_file.argtypes = [C.c_char_p, C.c_longlong, C.c_char_p]
    lib.rover_host_error.restype = C.c_char_p
    lib.rover_bundle_open_dir.argtypes = [C.c_char_p, C.c_int, C.POINTER(C.POINTER(Bundle))]
    lib.rover_bundle_close.argtypes = [C.POINTER(Bundle)]
    lib.rover_read_fvecs.argtypes = [C.c_char_p, C.c_int32, C.c_int32, C.POINTER(C.POINTER(C.c_float))]
    return lib


def _arr(ptr, ctype, count):
    return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(ctype)), shape=(count,)).copy()


def _open(host, d, verify=1):
    b = C.POINTER(Bundle)()
    rc = host.rover_bundle_open_dir(str(d).encode(), verify, C.byref(b))
    return rc, b, host.rover_host_error().decode()


def test_header_functions_are_exported(host):
    text = re.sub(r"/\*.*?\*/", "", (ROOT / "include" / "rover_host.h").read_text(), flags=re.S)
    names = set(re.findall(r"\b(rover_[a-z0-9_]+)\s*\(", text))
    assert len(names) >= 10
    for name in names:
        assert hasattr(host, name), name


@pytest.mark.parametrize("n", [0, 1, 55, 56, 63, 64, 65, 119, 120, 1000, 65537])
def test_sha256_matches_hashlib(host, n):
    data = np.random.default_rng(n).integers(0, 256, n, dtype=np.uint8).tobytes()
    out = C.create_string_buffer(32)
    host.rover_sha256(data, n, out)
    assert out.raw == hashlib.sha256(data).digest()


def test_sha256_file_with_offset(host, tmp_path):
    data = os.urandom(3 * 1024 * 1024 + 17)
    p = tmp_path / "blob"
    p.write_bytes(data)
    for off in (0, 1, 256, 4096):
        out = C.create_string_buffer(32)
        assert host.rover_sha256_file(str(p).encode(), off, out) == 0
        assert out.raw == hashlib.sha256(data[off:]).digest()


@pytest.mark.parametrize("name", PQ_FIXTURES + SQ_FIXTURES)
def test_bundle_loader_matches_python_reader(host, name):
    data, graph, b, _, _ = load_fixture(name)
    rc, cb, err = _open(host, GOLDEN / name)
    assert rc == 0, err
    try:
        x = cb.contents
        assert (x.n, x.dim, x.degree, x.graph_entry) == (data["n"], data["dim"], data["graph_degree"],
                                                         data["graph_entry"])
        assert np.array_equal(_arr(x.graph, C.c_int32, graph.size), graph.ravel())
        if data["method"] == "pq":
            md = b.meta
            assert x.method == 1 and (x.pq.m, x.pq.ks, x.pq.subdim, x.pq.code_bytes) == (md.m, md.ks, md.subdim,
                                                                                         md.code_bytes)
            assert bytes(x.index_uuid) == md.index_uuid
            assert np.array_equal(_arr(x.pq.codebook, C.c_float, b.codebook.size), b.codebook.ravel())
            assert np.array_equal(_arr(x.pq.codes, C.c_uint8, b.codes.size), b.codes.ravel())
            assert x.pq.residual_bits == b.residual_bits
            assert x.pq.residual_blocks_bytes == b.residual_blocks.size
            assert np.array_equal(_arr(x.pq.residual_blocks, C.c_uint8, b.residual_blocks.size), b.residual_blocks)
            assert np.array_equal(_arr(x.pq.residual_qparams, C.c_float, b.qparams.size), b.qparams.ravel())
        else:
            assert x.method == 0 and (x.sq.l1_bits, x.sq.residual_bits) == (b.l1_bits, b.residual_bits)
            assert np.float32(x.sq.l1_scale) == np.float32(b.l1_scale)
            assert np.float32(x.sq.l1_zero) == np.float32(b.l1_zero)
            assert np.array_equal(_arr(x.sq.l1_codes, C.c_uint8, b.l1.size), b.l1.ravel())
            assert np.array_equal(_arr(x.sq.residual_rows, C.c_uint8, b.residual_rows.size), b.residual_rows.ravel())
            assert np.array_equal(_arr(x.sq.residual_qparams, C.c_float, b.qparams.size), b.qparams.ravel())
    finally:
        host.rover_bundle_close(cb)


def _copy(tmp_path, name):
    d = tmp_path / name
    shutil.copytree(GOLDEN / name, d)
    return d


def _rerecord(d, key):
    """index.json updated for a member that was edited on purpose."""
    idx = json.loads((d / "index.json").read_text())
    p = d / idx["files"][key]["path"]
    idx["files"][key].update(bytes=p.stat().st_size, sha256=hashlib.sha256(p.read_bytes()).hexdigest())
    (d / "index.json").write_text(json.dumps(idx))


def test_bundle_loader_rejects_what_the_reference_rejects(host, tmp_path):
    # a changed member fails its index.json record
    d = _copy(tmp_path, "pq8_d64")
    raw = bytearray((d / "index.pqcodes").read_bytes())
    raw[300] ^= 1
    (d / "index.pqcodes").write_bytes(bytes(raw))
    rc, _, err = _open(host, d)
    assert rc != 0 and "Index member changed: pq_codes" in err
    # ... and, recorded anew, the payload checksum of its own header
    _rerecord(d, "pq_codes")
    rc, _, err = _open(host, d)
    assert rc != 0 and "payload checksum mismatch" in err
    # without verification the sizes still have to agree
    rc, b, err = _open(host, d, verify=0)
    assert rc == 0, err
    host.rover_bundle_close(b)
    # a graph with a self edge
    d = _copy(tmp_path / "g", "pq8_d64")
    raw = bytearray((d / "graph.rover").read_bytes())
    raw[16:20] = np.int32(0).tobytes()        # row 0, first neighbour = 0
    (d / "graph.rover").write_bytes(bytes(raw))
    _rerecord(d, "graph")
    rc, _, err = _open(host, d)
    assert rc != 0 and "self edge" in err
    # a member path outside the directory
    d = _copy(tmp_path / "p", "sq8_d32")
    idx = json.loads((d / "index.json").read_text())
    idx["files"]["l1"]["path"] = "../sq8_d32_twin/l1.bin"
    shutil.copytree(GOLDEN / "sq8_d32", tmp_path / "p" / "sq8_d32_twin")
    (d / "index.json").write_text(json.dumps(idx))
    rc, _, err = _open(host, d)
    assert rc != 0 and "Invalid index member l1" in err
    # a schema the reference does not know, and a malformed document
    d = _copy(tmp_path / "s", "sq4_d24")
    idx = json.loads((d / "index.json").read_text())
    (d / "index.json").write_text(json.dumps(dict(idx, schema="rover.index.v0")))
    rc, _, err = _open(host, d)
    assert rc != 0 and "Unsupported Rover index schema" in err
    (d / "index.json").write_text(json.dumps(idx)[:-3])
    rc, _, err = _open(host, d)
    assert rc != 0 and "JSON" in err
    # a reordered residual layout: the map is required (index_bundle.py:204),
    # and the reordered file itself is refused, not read in graph order
    (d / "index.json").write_text(json.dumps(dict(idx, residual_layout="b")))
    rc, _, err = _open(host, d)
    assert rc != 0 and "Index missing residual_map" in err
    idx["files"]["residual_map"] = dict(idx["files"]["graph"])
    (d / "index.json").write_text(json.dumps(dict(idx, residual_layout="b")))
    rc, _, err = _open(host, d)
    assert rc != 0 and "residual layout b" in err


def test_index_json_escapes_and_key_order(host, tmp_path):
    """index.json written with escaped characters and members in another
    order loads the same bundle."""
    d = _copy(tmp_path, "pq4_d24")
    idx = json.loads((d / "index.json").read_text())
    idx["dataset_note"] = "café \"quoted\" \\ tab\t \U0001F600"
    idx["files"] = dict(reversed(list(idx["files"].items())))
    (d / "index.json").write_text(json.dumps(idx, ensure_ascii=True, indent=3))
    rc, b, err = _open(host, d)
    assert rc == 0, err
    host.rover_bundle_close(b)


def test_fvecs_reader(host, tmp_path):
    from rover_b200 import bundle as B
    x = np.random.default_rng(0).normal(size=(7, 12)).astype(np.float32)
    p = tmp_path / "x.fvecs"
    B.write_fvecs(p, x)
    out = C.POINTER(C.c_float)()
    assert host.rover_read_fvecs(str(p).encode(), 5, 12, C.byref(out)) == 0
    assert np.array_equal(np.ctypeslib.as_array(out, shape=(5 * 12,)).reshape(5, 12), x[:5])
    assert host.rover_read_fvecs(str(p).encode(), 8, 12, C.byref(out)) != 0     # too few records
    assert host.rover_read_fvecs(str(p).encode(), 2, 11, C.byref(out)) != 0     # wrong dimension


def _rover(*args):
    return subprocess.run([str(ROVER), *args], capture_output=True, text=True, timeout=60)


def test_cli_options_and_checks(host):
    p = _rover("--help")
    assert p.returncode == 0
    ref_options = ["expand-count", "entry-points", "pool", "top-k", "refine-factor", "first-stage-factor", "index-dir",
                   "pq-prefix", "pq-book", "pq-codes", "pq-residual", "pq-qparams", "order-map", "graph-format",
                   "output", "metrics", "gt-k", "lanes", "cache-pages"]
    for o in ref_options:
        assert f"--{o} VALUE" in p.stdout, o
    base = ["search", "--n", "100", "--dim", "16", "--graph-degree", "8", "--nq", "1", "--query", "q", "--graph", "g"]
    p = _rover(*base, "--bogus", "1")
    assert p.returncode == 2 and "Unknown option: --bogus" in p.stderr
    p = _rover(*base, "--top-k", "0")
    assert p.returncode == 2 and "top-k 1..100; pool top-k..2000" in p.stderr
    p = _rover(*base, "--expand-count", "33")
    assert p.returncode == 2 and "invalid expand-count" in p.stderr
    p = _rover(*base, "--method", "pq", "--pq-m", "3")
    assert p.returncode == 2 and "PQ M must divide dim" in p.stderr
    p = _rover(*base, "--correction", "off", "--refine", "on")
    assert p.returncode == 2 and "outside this release" in p.stderr
    p = _rover("search", "--n", "100", "--dim", "16", "--graph-degree", "8", "--nq", "1")
    assert p.returncode == 2 and "search requires query, graph" in p.stderr
    p = _rover("build-index", "--n", "100", "--dim", "16", "--graph-degree", "8")
    assert p.returncode == 1 and "Construction" in p.stderr
    # a residual file in its own storage order is refused, not read as graph order
    p = _rover(*base, "--residual-map", "map.txt")
    assert p.returncode == 2 and "reordered residual files" in p.stderr
