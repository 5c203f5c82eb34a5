"""Rover index-bundle formats: readers, validators and writers.

The byte layouts are Rover's own, so a bundle prepared for the reference
loads here unchanged and vice versa:

* ``index.json`` -- schema ``rover.index.v1`` with a SHA-256 per member
  (reference tools/index_bundle.py:187-226, :270-345).
* graphs: ``rover`` (16-byte header ``<4i`` = 0x35314252, n, dim, degree,
  then int32 rows) and ``dense`` (raw int32 rows), -1 padded
  (tools/index_bundle.py:44-103).
* pure PQ: ``.pqbook`` / ``.pqcodes`` with the 256-byte ``PUREPQ01`` header
  (tools/build_pure_pq_index.py:67-97, src/dsp_demo/retrieval_pq_artifact.c),
  ``.pqresN`` (4096-byte header block, then 4096-byte residual blocks of
  ``4096 // code_bytes`` vectors, zero padded) and ``.pqresN.qparams``
  (256-byte header, then ``{f32 scale, f32 zero}`` per vector), both with the
  ``PQRES01`` header (tools/build_pure_pq_residual.py:46-66,
  src/dsp_demo/retrieval_pq_residual.c:216-246).
* SQ: ``l1.bin`` (32-byte ``L1MS`` header ``<IIiiiff4s`` + flat codes),
  ``residual.bin`` (4096-byte blocks, no header) and ``qparams.bin``
  (32-byte ``QPMS`` header ``<IIiiff8s`` + ``{scale, zero}`` per vector)
  (tools/encode_l1_residual.py:10-27, :140-212,
  src/dsp_demo/retrieval_rpc_demo_support.c:1053-1080).
"""
from __future__ import annotations

import hashlib
import json
import os
import struct
import uuid as uuidlib
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

SCHEMA = "rover.index.v1"
GRAPH_MAGIC = 0x35314252
BLOCK_BYTES = 4096

PQ_HEADER_BYTES = 256
PQ_MAGIC = b"PUREPQ01"
PQ_VERSION = (1, 1)
ENDIAN_MARKER = 0x01020304
PQ_KIND_CODEBOOK = 1
PQ_KIND_CODES = 2
TRAINER_SERVER_NUMPY = 2
SAMPLE_UNIFORM_STRIDE = 1

RES_MAGIC = b"PQRES01\0"
RES_VERSION = (1, 0)
RES_KIND_BLOCKS = 1
RES_KIND_QPARAMS = 2

L1_MAGIC = 0x314C4D53
L1_HEADER = struct.Struct("<IIiiiff4s")
QP_MAGIC = 0x51504D53
QP_HEADER = struct.Struct("<IIiiff8s")


class BundleError(ValueError):
    """A bundle member is missing, malformed or does not match its record."""


def sha256_file(path, offset: int = 0) -> str:
    digest = hashlib.sha256()
    with open(path, "rb") as f:
        f.seek(offset)
        for chunk in iter(lambda: f.read(8 << 20), b""):
            digest.update(chunk)
    return digest.hexdigest()


# ---------------------------------------------------------------- vectors

def write_fvecs(path, x: np.ndarray) -> None:
    x = np.ascontiguousarray(x, dtype="<f4")
    n, d = x.shape
    rec = np.empty((n, d + 1), dtype="<f4")
    rec.view("<i4")[:, 0] = d
    rec[:, 1:] = x
    rec.tofile(path)


def read_fvecs(path, count: int | None = None) -> np.ndarray:
    raw = np.fromfile(path, dtype="<i4")
    if raw.size == 0:
        raise BundleError(f"empty fvecs {path}")
    d = int(raw[0])
    if d <= 0 or raw.size % (d + 1):
        raise BundleError(f"malformed fvecs {path}")
    rec = raw.reshape(-1, d + 1)
    if np.any(rec[:, 0] != d):
        raise BundleError(f"inconsistent fvecs row dimension in {path}")
    out = rec[:, 1:].view("<f4")
    return np.ascontiguousarray(out[:count] if count is not None else out)


def write_ivecs(path, x: np.ndarray) -> None:
    x = np.ascontiguousarray(x, dtype="<i4")
    n, d = x.shape
    rec = np.empty((n, d + 1), dtype="<i4")
    rec[:, 0] = d
    rec[:, 1:] = x
    rec.tofile(path)


def read_ivecs(path, count: int | None = None) -> np.ndarray:
    raw = np.fromfile(path, dtype="<i4")
    d = int(raw[0])
    rec = raw.reshape(-1, d + 1)
    return np.ascontiguousarray(rec[:count, 1:] if count is not None else rec[:, 1:])


# ---------------------------------------------------------------- graph

def validate_graph(graph: np.ndarray, n: int) -> None:
    """Checks of tools/index_bundle.py:84-92: ids in [-1, n), no self edges,
    no duplicate edges."""
    for start in range(0, n, 8192):
        rows = graph[start:start + 8192]
        if np.any(rows < -1) or np.any(rows >= n):
            raise BundleError("Out-of-range graph neighbor")
        if np.any(rows == np.arange(start, start + len(rows))[:, None]):
            raise BundleError("Graph contains a self edge")
        ordered = np.sort(rows, axis=1)
        if np.any((ordered[:, 1:] >= 0) & (ordered[:, 1:] == ordered[:, :-1])):
            raise BundleError("Graph contains duplicate edges")


def write_graph(path, graph: np.ndarray, dim: int, kind: str = "rover") -> None:
    graph = np.ascontiguousarray(graph, dtype="<i4")
    n, degree = graph.shape
    with open(path, "wb") as f:
        if kind == "rover":
            f.write(struct.pack("<4i", GRAPH_MAGIC, n, dim, degree))
        elif kind != "dense":
            raise BundleError("graph kind must be rover or dense")
        f.write(graph.tobytes())


def read_graph(path, kind: str, n: int, degree: int, dim: int, validate: bool = True) -> np.ndarray:
    path = Path(path)
    if kind == "rover":
        if path.stat().st_size != 16 + n * degree * 4:
            raise BundleError("Rover graph size mismatch")
        with path.open("rb") as f:
            if f.read(16) != struct.pack("<4i", GRAPH_MAGIC, n, dim, degree):
                raise BundleError("Rover graph header mismatch")
        graph = np.fromfile(path, dtype="<i4", offset=16).reshape(n, degree)
    elif kind == "dense":
        if path.stat().st_size != n * degree * 4:
            raise BundleError("Dense graph size mismatch")
        graph = np.fromfile(path, dtype="<i4").reshape(n, degree)
    else:
        raise BundleError("Unknown graph format: " + kind)
    if validate:
        validate_graph(graph, n)
    return graph


# ---------------------------------------------------------------- pure PQ

def pq_code_bytes(m: int, ks: int) -> int:
    if ks == 16:
        return (m + 1) // 2
    if ks == 256:
        return m
    raise BundleError("Pure-PQ requires Ks=16 or Ks=256")


def residual_code_bytes(dim: int, bits: int) -> int:
    return (dim + 1) // 2 if bits == 4 else dim


@dataclass
class PqMeta:
    index_uuid: bytes
    num_vectors: int
    dim: int
    m: int
    ks: int
    subdim: int
    code_bytes: int
    trainer_kind: int = TRAINER_SERVER_NUMPY
    sample_strategy: int = SAMPLE_UNIFORM_STRIDE
    train_count: int = 1
    kmeans_iters: int = 1
    seed: int = 0
    dataset_fingerprint: bytes = bytes(32)
    layout_fingerprint: bytes = field(default_factory=lambda: hashlib.sha256(b"original").digest())


def _pq_header(kind: int, md: PqMeta, payload_bytes: int, payload_hash: bytes) -> bytes:
    h = bytearray(PQ_HEADER_BYTES)
    h[0:8] = PQ_MAGIC
    struct.pack_into("<HHIII", h, 8, PQ_VERSION[0], PQ_VERSION[1], PQ_HEADER_BYTES, kind, ENDIAN_MARKER)
    h[32:48] = md.index_uuid
    struct.pack_into("<QIIIIIIIIIIQII", h, 48, md.num_vectors, md.dim, md.m, md.ks, md.subdim,
                     md.code_bytes, 1, 1, 1, md.trainer_kind, md.sample_strategy,
                     md.train_count, md.kmeans_iters, md.seed)
    struct.pack_into("<Q", h, 112, payload_bytes)
    h[120:152] = payload_hash
    h[152:184] = md.dataset_fingerprint
    h[184:216] = md.layout_fingerprint
    return bytes(h)


def _parse_pq_header(raw: bytes, kind: int) -> tuple[PqMeta, int, bytes]:
    if len(raw) != PQ_HEADER_BYTES or raw[0:8] != PQ_MAGIC:
        raise BundleError("invalid Pure-PQ magic/header length")
    major, minor, hbytes, k, endian = struct.unpack_from("<HHIII", raw, 8)
    if major != PQ_VERSION[0] or minor > PQ_VERSION[1] or hbytes != PQ_HEADER_BYTES or endian != ENDIAN_MARKER:
        raise BundleError("unsupported Pure-PQ header")
    if k != kind:
        raise BundleError(f"artifact kind {k}, expected {kind}")
    (n, dim, m, ks, subdim, cb, metric, cdt, bdt, trainer, sample, train_count, iters,
     seed) = struct.unpack_from("<QIIIIIIIIIIQII", raw, 48)
    if (metric, cdt, bdt) != (1, 1, 1):
        raise BundleError("unsupported metric or payload dtype")
    md = PqMeta(bytes(raw[32:48]), n, dim, m, ks, subdim, cb, trainer, sample, train_count, iters,
                seed, bytes(raw[152:184]), bytes(raw[184:216]))
    if md.index_uuid == bytes(16) or n <= 0 or dim <= 0 or m <= 0 or subdim <= 0 or \
            m * subdim != dim or cb != pq_code_bytes(m, ks) or not 0 < train_count <= n or iters <= 0:
        raise BundleError("inconsistent Pure-PQ metadata")
    payload_bytes = struct.unpack_from("<Q", raw, 112)[0]
    return md, payload_bytes, bytes(raw[120:152])


def _res_header(kind: int, storage_header: int, md: PqMeta, bits: int, payload_bytes: int,
                payload_hash: bytes) -> bytes:
    rcb = residual_code_bytes(md.dim, bits)
    vpb = BLOCK_BYTES // rcb
    blocks = (md.num_vectors + vpb - 1) // vpb
    h = bytearray(PQ_HEADER_BYTES)
    h[0:8] = RES_MAGIC
    struct.pack_into("<HHIII", h, 8, RES_VERSION[0], RES_VERSION[1], storage_header, kind, ENDIAN_MARKER)
    struct.pack_into("<II", h, 24, bits, rcb)
    h[32:48] = md.index_uuid
    struct.pack_into("<QIIIIQ", h, 48, md.num_vectors, md.dim, BLOCK_BYTES, vpb, blocks, payload_bytes)
    h[80:112] = payload_hash
    h[112:144] = md.dataset_fingerprint
    h[144:176] = md.layout_fingerprint
    struct.pack_into("<I", h, 176, 8)
    return bytes(h)


def pack_residual_blocks(rows: np.ndarray) -> np.ndarray:
    """[n][code_bytes] rows -> block payload: 4096-byte blocks holding
    4096 // code_bytes rows each, zero padded (build_pure_pq_residual.py:161-213)."""
    n, rcb = rows.shape
    vpb = BLOCK_BYTES // rcb
    blocks = (n + vpb - 1) // vpb
    out = np.zeros((blocks, BLOCK_BYTES), dtype=np.uint8)
    padded = np.zeros((blocks * vpb, rcb), dtype=np.uint8)
    padded[:n] = rows
    out[:, :vpb * rcb] = padded.reshape(blocks, vpb * rcb)
    return out.reshape(-1)


def unpack_residual_blocks(payload: np.ndarray, n: int, rcb: int) -> np.ndarray:
    vpb = BLOCK_BYTES // rcb
    blocks = payload.reshape(-1, BLOCK_BYTES)[:, :vpb * rcb].reshape(-1, rcb)
    return np.ascontiguousarray(blocks[:n])


def write_pq_bundle(prefix, codebook: np.ndarray, codes: np.ndarray, residual_rows: np.ndarray | None,
                    qparams: np.ndarray | None, residual_bits: int = 8, *, train_count: int = 1,
                    kmeans_iters: int = 1, seed: int = 0, dataset_fingerprint: bytes | None = None,
                    index_uuid: bytes | None = None) -> PqMeta:
    """Write <prefix>.pqbook/.pqcodes/.pq.json and, with residuals,
    <prefix>.pqresN/.pqresN.qparams/.pqresN.json in the reference layouts."""
    codebook = np.ascontiguousarray(codebook, dtype="<f4")
    codes = np.ascontiguousarray(codes, dtype=np.uint8)
    m, ks, subdim = codebook.shape
    n = codes.shape[0]
    md = PqMeta(index_uuid or uuidlib.uuid4().bytes, n, m * subdim, m, ks, subdim,
                pq_code_bytes(m, ks), TRAINER_SERVER_NUMPY, SAMPLE_UNIFORM_STRIDE,
                max(1, min(train_count, n)), kmeans_iters, seed,
                dataset_fingerprint or bytes(32))
    if codes.shape[1] != md.code_bytes:
        raise BundleError("code byte count mismatch")
    prefix = str(prefix)
    for suffix, kind, payload in ((".pqbook", PQ_KIND_CODEBOOK, codebook.tobytes()),
                                  (".pqcodes", PQ_KIND_CODES, codes.tobytes())):
        digest = hashlib.sha256(payload).digest()
        with open(prefix + suffix, "wb") as f:
            f.write(_pq_header(kind, md, len(payload), digest))
            f.write(payload)
    manifest = dict(format="pure-pq-v1", artifact_source="server-numpy", index_uuid=md.index_uuid.hex(),
                    num_vectors=n, dim=md.dim, m=m, ks=ks, subdim=subdim,
                    code_bits=4 if ks == 16 else 8, code_bytes=md.code_bytes,
                    compression_x=(md.dim * 4) / md.code_bytes, metric="squared_l2",
                    train_count=md.train_count, kmeans_iters=kmeans_iters,
                    sample_strategy="uniform_stride", seed=seed,
                    dataset_fingerprint=md.dataset_fingerprint.hex(),
                    layout_id="original", layout_fingerprint=md.layout_fingerprint.hex(),
                    order_map_direction=None, order_map_fingerprint=None, order_map_path=None)
    with open(prefix + ".pq.json", "w") as f:
        json.dump(manifest, f, indent=2, sort_keys=True)
        f.write("\n")
    if residual_rows is not None:
        rows = np.ascontiguousarray(residual_rows, dtype=np.uint8)
        rcb = residual_code_bytes(md.dim, residual_bits)
        if rows.shape != (n, rcb):
            raise BundleError("residual rows shape mismatch")
        blocks = pack_residual_blocks(rows).tobytes()
        qp = np.ascontiguousarray(qparams, dtype="<f4").reshape(n, 2).tobytes()
        stem = f"{prefix}.pqres{residual_bits}"
        with open(stem, "wb") as f:
            f.write(_res_header(RES_KIND_BLOCKS, BLOCK_BYTES, md, residual_bits, len(blocks),
                                hashlib.sha256(blocks).digest()).ljust(BLOCK_BYTES, b"\0"))
            f.write(blocks)
        with open(stem + ".qparams", "wb") as f:
            f.write(_res_header(RES_KIND_QPARAMS, PQ_HEADER_BYTES, md, residual_bits, len(qp),
                                hashlib.sha256(qp).digest()))
            f.write(qp)
        vpb = BLOCK_BYTES // rcb
        with open(stem + ".json", "w") as f:
            json.dump(dict(format="pure-pq-residual-v1", index_uuid=md.index_uuid.hex(), num_vectors=n,
                           dim=md.dim, residual_bits=residual_bits, residual_code_bytes=rcb,
                           block_bytes=BLOCK_BYTES, vectors_per_block=vpb,
                           total_blocks=(n + vpb - 1) // vpb, blocks_payload_bytes=len(blocks),
                           blocks_payload_sha256=hashlib.sha256(blocks).hexdigest(),
                           qparams_payload_bytes=len(qp), qparams_payload_sha256=hashlib.sha256(qp).hexdigest(),
                           dataset_fingerprint=md.dataset_fingerprint.hex(),
                           layout_fingerprint=md.layout_fingerprint.hex(), layout_id="original",
                           order_map_direction=None, order_map_fingerprint=None),
                      f, indent=2, sort_keys=True)
            f.write("\n")
    return md


@dataclass
class PqBundle:
    meta: PqMeta
    codebook: np.ndarray        # [m][ks][subdim] f32
    codes: np.ndarray           # [n][code_bytes] u8
    residual_bits: int = 0
    residual_blocks: np.ndarray | None = None   # block payload, u8
    qparams: np.ndarray | None = None           # [n][2] f32

    @property
    def residual_code_bytes(self) -> int:
        return residual_code_bytes(self.meta.dim, self.residual_bits) if self.residual_bits else 0

    @property
    def vectors_per_block(self) -> int:
        return BLOCK_BYTES // self.residual_code_bytes if self.residual_bits else 0

    def residual_rows(self) -> np.ndarray:
        return unpack_residual_blocks(self.residual_blocks, self.meta.num_vectors, self.residual_code_bytes)


def read_pq_bundle(prefix, residual_bits: int = 0, verify_hashes: bool = True) -> PqBundle:
    """Load and validate a pure-PQ bundle the way retrieval_pq_artifacts_load
    (retrieval_pq_artifact.c:886-958) and retrieval_pq_residual_index_open
    (retrieval_pq_residual.c:716-835) accept it."""
    prefix = str(prefix)
    metas = []
    payloads = []
    for suffix, kind in ((".pqbook", PQ_KIND_CODEBOOK), (".pqcodes", PQ_KIND_CODES)):
        raw = Path(prefix + suffix).read_bytes()
        md, pbytes, phash = _parse_pq_header(raw[:PQ_HEADER_BYTES], kind)
        payload = raw[PQ_HEADER_BYTES:]
        if len(payload) != pbytes:
            raise BundleError(f"{prefix + suffix}: payload size mismatch")
        if verify_hashes and hashlib.sha256(payload).digest() != phash:
            raise BundleError(f"{prefix + suffix}: payload checksum mismatch")
        metas.append(md)
        payloads.append(payload)
    if metas[0] != metas[1]:
        raise BundleError("pqbook and pqcodes metadata mismatch")
    md = metas[0]
    codebook = np.frombuffer(payloads[0], dtype="<f4")
    if codebook.size != md.m * md.ks * md.subdim or not np.all(np.isfinite(codebook)):
        raise BundleError("invalid codebook payload")
    codes = np.frombuffer(payloads[1], dtype=np.uint8)
    if codes.size != md.num_vectors * md.code_bytes:
        raise BundleError("pqcodes payload size mismatch")
    bundle = PqBundle(md, codebook.reshape(md.m, md.ks, md.subdim).copy(),
                      codes.reshape(md.num_vectors, md.code_bytes).copy())
    if residual_bits:
        stem = f"{prefix}.pqres{residual_bits}"
        raw_blocks = Path(stem).read_bytes()
        raw_qp = Path(stem + ".qparams").read_bytes()
        for raw, kind, storage in ((raw_blocks, RES_KIND_BLOCKS, BLOCK_BYTES),
                                   (raw_qp, RES_KIND_QPARAMS, PQ_HEADER_BYTES)):
            h = raw[:PQ_HEADER_BYTES]
            if h[0:8] != RES_MAGIC:
                raise BundleError("invalid PQ residual header")
            major, minor, sh, k, endian = struct.unpack_from("<HHIII", h, 8)
            bits, rcb = struct.unpack_from("<II", h, 24)
            n, dim, bb, vpb, blocks, pbytes = struct.unpack_from("<QIIIIQ", h, 48)
            if (major, sh, k, endian) != (RES_VERSION[0], storage, kind, ENDIAN_MARKER) or minor > RES_VERSION[1] \
                    or struct.unpack_from("<I", h, 176)[0] != 8 or bits != residual_bits \
                    or rcb != residual_code_bytes(dim, bits) or bb != BLOCK_BYTES or vpb != BLOCK_BYTES // rcb \
                    or blocks != (n + vpb - 1) // vpb or n != md.num_vectors or dim != md.dim \
                    or bytes(h[32:48]) != md.index_uuid or bytes(h[112:144]) != md.dataset_fingerprint \
                    or bytes(h[144:176]) != md.layout_fingerprint:
                raise BundleError("PQ residual metadata mismatch")
            payload = raw[storage:]
            expect = blocks * BLOCK_BYTES if kind == RES_KIND_BLOCKS else n * 8
            if pbytes != expect or len(payload) != expect:
                raise BundleError("PQ residual payload size mismatch")
            if (verify_hashes or kind == RES_KIND_QPARAMS) and hashlib.sha256(payload).digest() != bytes(h[80:112]):
                raise BundleError("PQ residual checksum mismatch")
        bundle.residual_bits = residual_bits
        bundle.residual_blocks = np.frombuffer(raw_blocks[BLOCK_BYTES:], dtype=np.uint8).copy()
        bundle.qparams = np.frombuffer(raw_qp[PQ_HEADER_BYTES:], dtype="<f4").reshape(-1, 2).copy()
    return bundle


# ---------------------------------------------------------------- SQ

@dataclass
class SqBundle:
    num_vectors: int
    dim: int
    l1_bits: int
    l1_scale: float
    l1_zero: float
    l1: np.ndarray                  # [n][l1_code_bytes] u8
    residual_bits: int
    residual_rows: np.ndarray       # [n][residual_code_bytes] u8
    qparams: np.ndarray             # [n][2] f32

    @property
    def l1_code_bytes(self) -> int:
        return residual_code_bytes(self.dim, self.l1_bits)

    @property
    def residual_code_bytes(self) -> int:
        return residual_code_bytes(self.dim, self.residual_bits)


def write_sq_bundle(directory, b: SqBundle) -> dict:
    d = Path(directory)
    with open(d / "l1.bin", "wb") as f:
        f.write(L1_HEADER.pack(L1_MAGIC, 1, b.num_vectors, b.dim, b.l1_bits, float(b.l1_scale),
                               float(b.l1_zero), b"\0" * 4))
        f.write(np.ascontiguousarray(b.l1, dtype=np.uint8).tobytes())
    pack_residual_blocks(np.ascontiguousarray(b.residual_rows, dtype=np.uint8)).tofile(d / "residual.bin")
    with open(d / "qparams.bin", "wb") as f:
        f.write(QP_HEADER.pack(QP_MAGIC, 1, b.num_vectors, b.residual_bits, float(b.l1_scale),
                               float(b.l1_zero), b"\0" * 8))
        f.write(np.ascontiguousarray(b.qparams, dtype="<f4").tobytes())
    return {k: d / f"{k}.bin" for k in ("l1", "residual", "qparams")}


def read_sq_bundle(l1_path, residual_path, qparams_path) -> SqBundle:
    """Readers for the L1MS / QPMS / residual block files
    (retrieval_demo_load_l1_and_qparams_from_disk,
    retrieval_rpc_demo_support.c:1968)."""
    raw = Path(l1_path).read_bytes()
    magic, ver, n, dim, bits, scale, zero, _ = L1_HEADER.unpack_from(raw, 0)
    if magic != L1_MAGIC or ver != 1 or n <= 0 or dim <= 0 or bits not in (4, 8):
        raise BundleError("invalid L1 code file header")
    cb = residual_code_bytes(dim, bits)
    if len(raw) != L1_HEADER.size + n * cb:
        raise BundleError("L1 code file size mismatch")
    l1 = np.frombuffer(raw[L1_HEADER.size:], dtype=np.uint8).reshape(n, cb).copy()
    raw = Path(qparams_path).read_bytes()
    qmagic, qver, qn, rbits, qscale, qzero, _ = QP_HEADER.unpack_from(raw, 0)
    if qmagic != QP_MAGIC or qver != 1 or qn != n or rbits not in (4, 8) or \
            np.float32(qscale) != np.float32(scale) or np.float32(qzero) != np.float32(zero):
        raise BundleError("invalid qparams file header")
    if len(raw) != QP_HEADER.size + n * 8:
        raise BundleError("qparams file size mismatch")
    qparams = np.frombuffer(raw[QP_HEADER.size:], dtype="<f4").reshape(n, 2).copy()
    rcb = residual_code_bytes(dim, rbits)
    payload = np.fromfile(residual_path, dtype=np.uint8)
    vpb = BLOCK_BYTES // rcb
    if payload.size != ((n + vpb - 1) // vpb) * BLOCK_BYTES:
        raise BundleError("residual block file size mismatch")
    rows = unpack_residual_blocks(payload, n, rcb)
    return SqBundle(n, dim, bits, float(np.float32(scale)), float(np.float32(zero)), l1, rbits, rows, qparams)


# ---------------------------------------------------------------- index.json

def member_record(path, root) -> dict:
    path, root = Path(path), Path(root)
    return dict(path=str(path.relative_to(root)), bytes=path.stat().st_size, sha256=sha256_file(path))


def write_index_json(directory, data: dict) -> Path:
    path = Path(directory) / "index.json"
    with open(path, "w") as f:
        json.dump(data, f, indent=2)
        f.write("\n")
    return path


def validate_index(directory, third: bool = False, require_graph: bool = True,
                   verify_hashes: bool = True) -> dict:
    """tools/index_bundle.py:187-226 (validate)."""
    directory = Path(directory).resolve()
    data = json.loads((directory / "index.json").read_text())
    if data.get("schema") != SCHEMA:
        raise BundleError("Unsupported Rover index schema")
    if data.get("method") not in ("sq", "pq") or not 0 < data["dim"] <= 1024 or \
            not 0 < data["graph_degree"] < data["n"] <= 2147483647:
        raise BundleError("Invalid index method or dimensions")
    if data["residual_bits"] not in (4, 8) or \
            data.get("sq_bits" if data["method"] == "sq" else "pq_bits") not in (4, 8):
        raise BundleError("Index bits must be 4 or 8")
    required = ["l1", "residual", "qparams"] if data["method"] == "sq" else \
        ["pq_book", "pq_codes", "pq_residual", "pq_qparams", "pq_manifest", "pq_residual_manifest"]
    if require_graph:
        required.append("graph")
    if third:
        required.append("error4")
    if data.get("reordered"):
        required.append("order_map")
    if data.get("residual_layout", "a") != "a":
        required.append("residual_map")
    for key in required:
        if key not in data["files"]:
            raise BundleError("Index missing " + key)
    names = set()
    for key, item in data["files"].items():
        if key == "error4" and not third:
            continue
        path = (directory / item["path"]).resolve()
        if Path(item["path"]).is_absolute() or not path.is_relative_to(directory) or not path.is_file():
            raise BundleError("Invalid index member " + key)
        if path.name in names:
            raise BundleError("Colliding index member names")
        names.add(path.name)
        if path.stat().st_size != item["bytes"] or (verify_hashes and sha256_file(path) != item["sha256"]):
            raise BundleError("Index member changed: " + key)
    if data["method"] == "pq":
        suffix = f".pqres{data['residual_bits']}"
        expect = dict(pq_book="index.pqbook", pq_codes="index.pqcodes", pq_manifest="index.pq.json",
                      pq_residual="index" + suffix, pq_qparams="index" + suffix + ".qparams",
                      pq_residual_manifest="index" + suffix + ".json")
        if any(Path(data["files"][k]["path"]).name != v for k, v in expect.items()):
            raise BundleError("PQ bundle filenames must use the index prefix")
    return data


def write_pq_index_dir(directory, graph: np.ndarray, graph_entry: int, codebook, codes, residual_rows,
                       qparams, residual_bits: int, **kw) -> dict:
    """A complete ``rover.index.v1`` PQ bundle directory (graph.rover +
    index.* members + index.json), as tools/index_bundle.py:270-345 lays it out."""
    d = Path(directory)
    d.mkdir(parents=True, exist_ok=True)
    n, degree = graph.shape
    dim = codebook.shape[0] * codebook.shape[2]
    write_graph(d / "graph.rover", graph, dim)
    md = write_pq_bundle(d / "index", codebook, codes, residual_rows, qparams, residual_bits, **kw)
    files = {"graph": member_record(d / "graph.rover", d)}
    suffix = f".pqres{residual_bits}"
    for key, ext in (("pq_book", ".pqbook"), ("pq_codes", ".pqcodes"), ("pq_manifest", ".pq.json"),
                     ("pq_residual", suffix), ("pq_qparams", suffix + ".qparams"),
                     ("pq_residual_manifest", suffix + ".json")):
        files[key] = member_record(d / ("index" + ext), d)
    data = dict(schema=SCHEMA, n=n, dim=dim, graph_degree=degree, method="pq", residual_bits=residual_bits,
                third_residual=False, reordered=False, layout="original",
                layout_hash=hashlib.sha256(b"original").hexdigest(), graph_format="rover",
                graph_entry=int(graph_entry), files=files, raw_sha256="",
                pq_bits=4 if md.ks == 16 else 8, pq_m=md.m, train_samples=md.train_count,
                train_iters=md.kmeans_iters, seed=md.seed, residual_layout="a")
    write_index_json(d, data)
    return data


def write_sq_index_dir(directory, graph: np.ndarray, graph_entry: int, b: SqBundle) -> dict:
    d = Path(directory)
    d.mkdir(parents=True, exist_ok=True)
    n, degree = graph.shape
    write_graph(d / "graph.rover", graph, b.dim)
    paths = write_sq_bundle(d, b)
    files = {"graph": member_record(d / "graph.rover", d)}
    for key, p in paths.items():
        files[key] = member_record(p, d)
    data = dict(schema=SCHEMA, n=n, dim=b.dim, graph_degree=degree, method="sq",
                residual_bits=b.residual_bits, third_residual=False, reordered=False, layout="original",
                layout_hash=hashlib.sha256(b"original").hexdigest(), graph_format="rover",
                graph_entry=int(graph_entry), files=files, raw_sha256="", residual_layout="a",
                sq_bits=b.l1_bits)
    write_index_json(d, data)
    return data


def load_index_dir(directory, verify_hashes: bool = True):
    """Validate ``index.json`` and load the graph plus the PQ or SQ members.
    Returns (data, graph, bundle)."""
    directory = Path(directory)
    data = validate_index(directory, verify_hashes=verify_hashes)
    graph = read_graph(directory / data["files"]["graph"]["path"], data.get("graph_format", "rover"),
                       data["n"], data["graph_degree"], data["dim"], validate=verify_hashes)
    if data["method"] == "pq":
        prefix = directory / "index"
        bundle = read_pq_bundle(prefix, data["residual_bits"], verify_hashes=verify_hashes)
    else:
        f = data["files"]
        bundle = read_sq_bundle(directory / f["l1"]["path"], directory / f["residual"]["path"],
                                directory / f["qparams"]["path"])
    return data, graph, bundle


def fsync_dir(path) -> None:
    fd = os.open(path, os.O_RDONLY)
    try:
        os.fsync(fd)
    finally:
        os.close(fd)
