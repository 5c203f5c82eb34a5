"""ctypes bindings for the oracle libraries -- TEST INFRASTRUCTURE ONLY.

* ``Reference``: oracle/_ref/libref_harness.so, the unmodified reference
  sources compiled here (see oracle/Makefile) plus a thread fan-out driver.
* ``Port``: oracle/_build/liboracle.so, this project's C restatement.

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of bench.py
import this module; the product path never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_LIB = HERE / "_ref" / "libref_harness.so"
PORT_LIB = HERE / "_build" / "liboracle.so"

_i32p = C.POINTER(C.c_int32)
_f32p = C.POINTER(C.c_float)
_u8p = C.POINTER(C.c_uint8)
_u64p = C.POINTER(C.c_uint64)


def _p(a, t):
    return None if a is None else a.ctypes.data_as(t)


def build(reference_dir: str | None = None) -> None:
    """Compile the port always, and the reference when its sources exist:
    at ``reference_dir``, else $ROVER_REFERENCE, else the checkout location
    the Makefile names (its ``ref-if-present`` target skips a missing one)."""
    subprocess.run(["make", "-s", "-C", str(HERE), "port"], check=True)
    ref = reference_dir or os.environ.get("ROVER_REFERENCE")
    extra = [f"REF={Path(ref).resolve()}"] if ref else []
    subprocess.run(["make", "-s", "-C", str(HERE), "ref-if-present", *extra], check=True)


def reference_available() -> bool:
    return REF_LIB.is_file()


def port_available() -> bool:
    return PORT_LIB.is_file()


class _PqConfig(C.Structure):
    """RetrievalPqConfig (retrieval_pq_core.h:10-17)."""
    _fields_ = [("m", C.c_int), ("ks", C.c_int), ("subdim", C.c_int), ("dim", C.c_int), ("train_max", C.c_int),
                ("kmeans_iters", C.c_int)]


class Reference:
    """The reference's own functions, driven in batches."""

    def __init__(self):
        self.lib = C.CDLL(str(REF_LIB))
        L = self.lib
        L.ref_pq_open.argtypes = [C.c_char_p, C.c_int, C.c_int, C.POINTER(C.c_void_p)]
        L.ref_pq_close.argtypes = [C.c_void_p]
        L.ref_pq_info.argtypes = [C.c_void_p, _i32p]
        L.ref_pq_lut.argtypes = [C.c_void_p, _f32p, _f32p]
        L.ref_pq_adc.argtypes = [C.c_void_p, _f32p, _i32p, C.c_int, _f32p]
        L.ref_pq_residual_eval.argtypes = [C.c_void_p, _f32p, _i32p, C.c_int, _f32p]
        L.ref_pq_residual_decode.argtypes = [C.c_void_p, C.c_int, _f32p]
        L.ref_pq_seed_ids.argtypes = [C.c_int, C.c_int, C.c_int, C.c_uint, _i32p]
        L.ref_pq_search_batch.argtypes = [C.c_void_p, _i32p, C.c_int, C.c_int, _f32p, C.c_int, _i32p,
                                          C.c_int, C.c_int, C.c_uint, C.c_int, C.c_int, C.c_int, C.c_int,
                                          _i32p, _f32p, C.c_int, _i32p, _i32p, _f32p, C.c_int, _i32p, _u64p]
        L.ref_sq_open.argtypes = [C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, _u8p, C.c_int, _u8p,
                                  _f32p, C.POINTER(C.c_void_p)]
        L.ref_sq_close.argtypes = [C.c_void_p]
        L.ref_sq_quantize.argtypes = [C.c_void_p, _f32p, _u8p]
        L.ref_sq_coarse.argtypes = [C.c_void_p, _f32p, _i32p, C.c_int, _f32p]
        L.ref_sq_exact.argtypes = [C.c_void_p, _f32p, _i32p, C.c_int, _f32p]
        L.ref_sq_sqmd_batch.argtypes = [C.c_void_p, _i32p, C.c_int, C.c_int, _f32p, C.c_int, _i32p, C.c_int,
                                        C.c_int, C.c_uint, C.c_int, C.c_int, C.c_int, _i32p, _f32p, C.c_int,
                                        _i32p]
        L.ref_refine_batch.argtypes = [C.c_int, C.c_void_p, _f32p, C.c_int, C.c_int, _i32p, _f32p, C.c_int,
                                       _i32p, C.c_int, _i32p]
        L.ref_dsp_search_batch.argtypes = [C.c_int, _i32p, C.c_int, C.c_int, C.c_int, _u8p, C.c_int, C.c_int,
                                           C.c_float, C.c_float, _f32p, C.c_int, _i32p, C.c_int, C.c_int,
                                           C.c_int, C.c_int, _i32p, _f32p, C.c_int, _i32p]

    # -- PQ training and encoding (retrieval_pq_core.c:97-268, called directly)
    def pq_train(self, vectors, m: int, ks: int, iters: int):
        x = np.ascontiguousarray(vectors, dtype=np.float32)
        n, dim = x.shape
        cfg = _PqConfig(m, ks, dim // m, dim, n, iters)
        book = np.zeros((m, ks, dim // m), np.float32)
        self.lib.retrieval_pq_train.argtypes = [_f32p, C.c_int, C.POINTER(_PqConfig), _f32p]
        rc = self.lib.retrieval_pq_train(_p(x, _f32p), n, C.byref(cfg), _p(book, _f32p))
        if rc != 0:
            raise RuntimeError(f"retrieval_pq_train failed: {rc}")
        return book

    def pq_encode(self, vectors, book):
        x = np.ascontiguousarray(vectors, dtype=np.float32)
        b = np.ascontiguousarray(book, dtype=np.float32)
        m, ks, subdim = b.shape
        cfg = _PqConfig(m, ks, subdim, m * subdim, 0, 1)
        cb = (m + 1) // 2 if ks <= 16 else m
        codes = np.zeros((x.shape[0], cb), np.uint8)
        self.lib.retrieval_pq_encode_batch.argtypes = [_f32p, C.c_int, _f32p, C.POINTER(_PqConfig), _u8p]
        rc = self.lib.retrieval_pq_encode_batch(_p(x, _f32p), x.shape[0], _p(b, _f32p), C.byref(cfg),
                                                _p(codes, _u8p))
        if rc != 0:
            raise RuntimeError(f"retrieval_pq_encode_batch failed: {rc}")
        return codes

    # -- PQ
    def pq_open(self, prefix, residual_bits: int, chunk_vectors: int = 262144):
        h = C.c_void_p()
        rc = self.lib.ref_pq_open(str(prefix).encode(), residual_bits, chunk_vectors, C.byref(h))
        if rc != 0:
            raise RuntimeError(f"ref_pq_open failed: {rc}")
        return h

    def pq_close(self, h):
        self.lib.ref_pq_close(h)

    def pq_lut(self, h, query, m, ks):
        q = np.ascontiguousarray(query, dtype=np.float32)
        out = np.empty(m * ks, dtype=np.float32)
        if self.lib.ref_pq_lut(h, _p(q, _f32p), _p(out, _f32p)) != 0:
            raise RuntimeError("ref_pq_lut failed")
        return out

    def pq_adc(self, h, lut, ids):
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        out = np.empty(len(ids), dtype=np.float32)
        rc = self.lib.ref_pq_adc(h, _p(np.ascontiguousarray(lut, dtype=np.float32), _f32p),
                                 _p(ids, _i32p), len(ids), _p(out, _f32p))
        if rc != 0:
            raise RuntimeError("ref_pq_adc failed")
        return out

    def pq_residual_eval(self, h, query, ids):
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        out = np.empty(len(ids), dtype=np.float32)
        q = np.ascontiguousarray(query, dtype=np.float32)
        if self.lib.ref_pq_residual_eval(h, _p(q, _f32p), _p(ids, _i32p), len(ids), _p(out, _f32p)) != 0:
            raise RuntimeError("ref_pq_residual_eval failed")
        return out

    def pq_seed_ids(self, n, entry_count, graph_entry, seed=42):
        out = np.empty(max(1, min(entry_count, n)), dtype=np.int32)
        c = self.lib.ref_pq_seed_ids(n, entry_count, graph_entry, seed, _p(out, _i32p))
        return out[:c]

    def pq_search(self, h, graph, graph_entry, queries, pool_sizes, entry_points, expand_count,
                  correction=1, refine_budget=0, top_k=10, threads=1, seed=42):
        graph = np.ascontiguousarray(graph, dtype=np.int32)
        queries = np.ascontiguousarray(queries, dtype=np.float32)
        nq = queries.shape[0]
        pools = np.ascontiguousarray(np.broadcast_to(np.asarray(pool_sizes, dtype=np.int32), (nq,)))
        stride = int(pools.max())
        pool_ids = np.full((nq, stride), -1, dtype=np.int32)
        pool_d = np.zeros((nq, stride), dtype=np.float32)
        pool_c = np.zeros(nq, dtype=np.int32)
        out_ids = np.full((nq, top_k), -1, dtype=np.int32)
        out_d = np.zeros((nq, top_k), dtype=np.float32)
        out_c = np.zeros(nq, dtype=np.int32)
        stats = np.zeros((nq, 4), dtype=np.uint64)
        rc = self.lib.ref_pq_search_batch(h, _p(graph, _i32p), graph.shape[1], graph_entry, _p(queries, _f32p),
                                          nq, _p(pools, _i32p), entry_points, expand_count, seed, correction,
                                          refine_budget, top_k, threads, _p(pool_ids, _i32p), _p(pool_d, _f32p),
                                          stride, _p(pool_c, _i32p), _p(out_ids, _i32p), _p(out_d, _f32p),
                                          top_k, _p(out_c, _i32p), _p(stats, _u64p))
        if rc != 0:
            raise RuntimeError(f"ref_pq_search_batch failed at query {rc - 1}")
        return dict(pool_ids=pool_ids, pool_dists=pool_d, pool_counts=pool_c, ids=out_ids, dists=out_d,
                    counts=out_c, stats=stats)

    # -- SQ
    def sq_open(self, b):
        """b: rover_b200.bundle.SqBundle (arrays are kept alive on the handle)."""
        h = C.c_void_p()
        keep = (np.ascontiguousarray(b.l1, dtype=np.uint8), np.ascontiguousarray(b.residual_rows, dtype=np.uint8),
                np.ascontiguousarray(b.qparams, dtype=np.float32))
        rc = self.lib.ref_sq_open(b.num_vectors, b.dim, b.l1_bits, b.l1_scale, b.l1_zero, _p(keep[0], _u8p),
                                  b.residual_bits, _p(keep[1], _u8p), _p(keep[2], _f32p), C.byref(h))
        if rc != 0:
            raise RuntimeError("ref_sq_open failed")
        return (h, keep, b)

    def sq_close(self, hs):
        self.lib.ref_sq_close(hs[0])

    def sq_quantize(self, hs, query):
        q = np.ascontiguousarray(query, dtype=np.float32)
        out = np.empty(q.shape[0], dtype=np.uint8)
        if self.lib.ref_sq_quantize(hs[0], _p(q, _f32p), _p(out, _u8p)) != 0:
            raise RuntimeError("ref_sq_quantize failed")
        return out

    def sq_coarse(self, hs, query, ids):
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        q = np.ascontiguousarray(query, dtype=np.float32)
        out = np.empty(len(ids), dtype=np.float32)
        if self.lib.ref_sq_coarse(hs[0], _p(q, _f32p), _p(ids, _i32p), len(ids), _p(out, _f32p)) != 0:
            raise RuntimeError("ref_sq_coarse failed")
        return out

    def sq_exact(self, hs, query, ids):
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        q = np.ascontiguousarray(query, dtype=np.float32)
        out = np.empty(len(ids), dtype=np.float32)
        self.lib.ref_sq_exact(hs[0], _p(q, _f32p), _p(ids, _i32p), len(ids), _p(out, _f32p))
        return out

    def sqmd_search(self, hs, graph, graph_entry, queries, pool_sizes, entry_points, expand_count,
                    correction=1, lanes=4, threads=1, seed=42, out_cap=None):
        graph = np.ascontiguousarray(graph, dtype=np.int32)
        queries = np.ascontiguousarray(queries, dtype=np.float32)
        nq = queries.shape[0]
        pools = np.ascontiguousarray(np.broadcast_to(np.asarray(pool_sizes, dtype=np.int32), (nq,)))
        stride = out_cap or int(pools.max())
        ids = np.full((nq, stride), -1, dtype=np.int32)
        d = np.zeros((nq, stride), dtype=np.float32)
        c = np.zeros(nq, dtype=np.int32)
        rc = self.lib.ref_sq_sqmd_batch(hs[0], _p(graph, _i32p), graph.shape[1], graph_entry, _p(queries, _f32p),
                                        nq, _p(pools, _i32p), entry_points, expand_count, seed, lanes, correction,
                                        threads, _p(ids, _i32p), _p(d, _f32p), stride, _p(c, _i32p))
        if rc != 0:
            raise RuntimeError(f"ref_sq_sqmd_batch failed at query {rc - 1}")
        return dict(ids=ids, dists=d, counts=c)

    def refine(self, kind, handle, queries, cand_ids, cand_dists, cand_counts, top_k):
        queries = np.ascontiguousarray(queries, dtype=np.float32)
        ids = np.array(cand_ids, dtype=np.int32, copy=True)
        d = np.array(cand_dists, dtype=np.float32, copy=True)
        counts = np.ascontiguousarray(cand_counts, dtype=np.int32)
        out_c = np.zeros(len(counts), dtype=np.int32)
        h = handle[0] if isinstance(handle, tuple) else handle
        rc = self.lib.ref_refine_batch(kind, h, _p(queries, _f32p), queries.shape[1], queries.shape[0],
                                       _p(ids, _i32p), _p(d, _f32p), ids.shape[1], _p(counts, _i32p), top_k,
                                       _p(out_c, _i32p))
        if rc != 0:
            raise RuntimeError(f"ref_refine_batch failed: {rc}")
        return ids[:, :top_k], d[:, :top_k], out_c

    def dsp_search(self, b, graph, graph_entry, queries, pool_sizes, entry_points, expand_count, num_out,
                   threads=1):
        graph = np.ascontiguousarray(graph, dtype=np.int32)
        queries = np.ascontiguousarray(queries, dtype=np.float32)
        l1 = np.ascontiguousarray(b.l1, dtype=np.uint8)
        nq = queries.shape[0]
        pools = np.ascontiguousarray(np.broadcast_to(np.asarray(pool_sizes, dtype=np.int32), (nq,)))
        ids = np.full((nq, num_out), -1, dtype=np.int32)
        d = np.zeros((nq, num_out), dtype=np.float32)
        c = np.zeros(nq, dtype=np.int32)
        rc = self.lib.ref_dsp_search_batch(b.l1_bits, _p(graph, _i32p), graph.shape[0], graph.shape[1], graph_entry,
                                           _p(l1, _u8p), l1.size, b.dim, b.l1_scale, b.l1_zero, _p(queries, _f32p),
                                           nq, _p(pools, _i32p), entry_points, expand_count, num_out, threads,
                                           _p(ids, _i32p), _p(d, _f32p), num_out, _p(c, _i32p))
        if rc != 0:
            raise RuntimeError(f"ref_dsp_search_batch failed: {rc}")
        return dict(ids=ids, dists=d, counts=c)


class _PqIndex(C.Structure):
    _fields_ = [("graph", _i32p), ("n", C.c_int32), ("degree", C.c_int32), ("dim", C.c_int32),
                ("codes", _u8p), ("codebook", _f32p), ("m", C.c_int32), ("ks", C.c_int32),
                ("subdim", C.c_int32), ("code_bytes", C.c_int32), ("residual", _u8p),
                ("residual_bits", C.c_int32), ("residual_code_bytes", C.c_int32),
                ("vectors_per_block", C.c_int32), ("qparams", _f32p)]


class _SqIndex(C.Structure):
    _fields_ = [("graph", _i32p), ("n", C.c_int32), ("degree", C.c_int32), ("dim", C.c_int32),
                ("l1", _u8p), ("l1_bits", C.c_int32), ("l1_code_bytes", C.c_int32),
                ("l1_scale", C.c_float), ("l1_zero", C.c_float), ("residual", _u8p),
                ("residual_bits", C.c_int32), ("residual_code_bytes", C.c_int32), ("qparams", _f32p)]


class _Error4(C.Structure):
    _fields_ = [("qparams", _f32p), ("blocks", _u8p), ("code_bytes", C.c_int32),
                ("vectors_per_block", C.c_int32)]


class _SplitQuery(C.Structure):
    _fields_ = [("q", C.c_uint8 * 1024), ("sum_q", C.c_uint64)]


def read_error4(path, n: int, dim: int):
    """The ERROR4 artifact's payload (256-byte header skipped): per-row
    {scale, zero} and the 4096-byte code blocks."""
    raw = np.fromfile(path, dtype=np.uint8)
    qp = raw[256:256 + 8 * n].view(np.float32).reshape(n, 2).copy()
    blocks = raw[256 + 8 * n:].copy()
    return qp, blocks, (dim + 1) // 2, 4096 // ((dim + 1) // 2)


def read_bias(path, n: int):
    """The split-distance bias payload (64-byte header skipped)."""
    return np.fromfile(path, dtype=np.uint8)[64:64 + 4 * n].view(np.float32).copy()


class Port:
    """This project's C restatement of the path (oracle/rover_oracle.c)."""

    def __init__(self):
        self.lib = C.CDLL(str(PORT_LIB))
        L = self.lib
        L.oracle_pq_build_lut.argtypes = [C.POINTER(_PqIndex), _f32p, _f32p]
        L.oracle_pq_adc.argtypes = [C.POINTER(_PqIndex), _f32p, _i32p, C.c_int, _f32p]
        L.oracle_pq_residual_eval.argtypes = [C.POINTER(_PqIndex), _f32p, _i32p, C.c_int, _f32p]
        L.oracle_pq_decode.argtypes = [C.POINTER(_PqIndex), C.c_int, _f32p]
        L.oracle_pq_seed_ids.argtypes = [C.c_int, C.c_int, C.c_int, C.c_uint32, _i32p]
        L.oracle_pq_search_batch.argtypes = [C.POINTER(_PqIndex), _f32p, C.c_int, _i32p, C.c_int, C.c_int,
                                             C.c_uint32, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _i32p,
                                             _f32p, C.c_int, _i32p, _i32p, _f32p, C.c_int, _i32p, _u64p]
        L.oracle_sq_quantize.argtypes = [C.POINTER(_SqIndex), _f32p, _u8p]
        L.oracle_sq_coarse.argtypes = [C.POINTER(_SqIndex), _u8p, C.c_int]
        L.oracle_sq_coarse.restype = C.c_float
        L.oracle_sq_exact.argtypes = [C.POINTER(_SqIndex), _f32p, C.c_int]
        L.oracle_sq_exact.restype = C.c_float
        L.oracle_sq_seed_ids.argtypes = [C.c_int, C.c_int, C.c_int, C.c_uint32, _i32p, C.c_int]
        L.oracle_sqmd_search.argtypes = [C.POINTER(_SqIndex), _f32p, C.c_int, C.c_int, C.c_uint32, C.c_int,
                                         C.c_int, C.c_int, _i32p, _f32p, C.c_int, _u64p]
        L.oracle_dsp_search.argtypes = [C.POINTER(_SqIndex), _f32p, C.c_int, C.c_int, C.c_int, C.c_int,
                                        C.c_int, _i32p, _f32p]
        L.oracle_refine.argtypes = [C.c_int, C.c_void_p, _f32p, _i32p, C.c_int, C.c_int, _i32p, _f32p]
        L.oracle_sq_rerank.argtypes = [C.POINTER(_SqIndex), _f32p, _i32p, _f32p, C.c_int, C.c_int, _i32p, _f32p]
        L.oracle_refine_ex.argtypes = [C.c_int, C.c_void_p, C.POINTER(_Error4), _f32p, _i32p, C.c_int, C.c_int,
                                       _i32p, _f32p]
        L.oracle_split_query.argtypes = [C.POINTER(_SqIndex), _f32p, C.POINTER(_SplitQuery)]
        for f in ("oracle_split_coarse",):
            getattr(L, f).argtypes = [C.POINTER(_SqIndex), C.POINTER(_SplitQuery), C.c_int]
            getattr(L, f).restype = C.c_float
        for f in ("oracle_split_delta", "oracle_split_distance"):
            getattr(L, f).argtypes = [C.POINTER(_SqIndex), _f32p, C.POINTER(_SplitQuery), C.c_int]
            getattr(L, f).restype = C.c_float
        L.oracle_sqmd_search_split.argtypes = [C.POINTER(_SqIndex), _f32p, _f32p, C.c_int, C.c_int, C.c_uint32,
                                               C.c_int, C.c_int, _i32p, _f32p, C.c_int, _u64p]

    def pq_index(self, graph, bundle):
        """(struct, keepalive) for a rover_b200.bundle.PqBundle + graph."""
        g = np.ascontiguousarray(graph, dtype=np.int32)
        codes = np.ascontiguousarray(bundle.codes, dtype=np.uint8)
        book = np.ascontiguousarray(bundle.codebook, dtype=np.float32)
        res = np.ascontiguousarray(bundle.residual_blocks if bundle.residual_bits else np.zeros(1, np.uint8))
        qp = np.ascontiguousarray(bundle.qparams if bundle.residual_bits else np.zeros((1, 2), np.float32),
                                  dtype=np.float32)
        md = bundle.meta
        s = _PqIndex(_p(g, _i32p), md.num_vectors, g.shape[1], md.dim, _p(codes, _u8p), _p(book, _f32p), md.m,
                     md.ks, md.subdim, md.code_bytes, _p(res, _u8p), bundle.residual_bits,
                     bundle.residual_code_bytes, bundle.vectors_per_block, _p(qp, _f32p))
        return s, (g, codes, book, res, qp)

    def sq_index(self, graph, b):
        g = np.ascontiguousarray(graph, dtype=np.int32)
        l1 = np.ascontiguousarray(b.l1, dtype=np.uint8)
        res = np.ascontiguousarray(b.residual_rows, dtype=np.uint8)
        qp = np.ascontiguousarray(b.qparams, dtype=np.float32)
        s = _SqIndex(_p(g, _i32p), b.num_vectors, g.shape[1], b.dim, _p(l1, _u8p), b.l1_bits, b.l1_code_bytes,
                     b.l1_scale, b.l1_zero, _p(res, _u8p), b.residual_bits, b.residual_code_bytes, _p(qp, _f32p))
        return s, (g, l1, res, qp)

    def pq_lut(self, ix, query):
        s = ix[0]
        q = np.ascontiguousarray(query, dtype=np.float32)
        out = np.empty(s.m * s.ks, dtype=np.float32)
        if self.lib.oracle_pq_build_lut(C.byref(s), _p(q, _f32p), _p(out, _f32p)) != 0:
            raise RuntimeError("oracle_pq_build_lut failed")
        return out

    def pq_adc(self, ix, lut, ids):
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        out = np.empty(len(ids), dtype=np.float32)
        if self.lib.oracle_pq_adc(C.byref(ix[0]), _p(np.ascontiguousarray(lut, dtype=np.float32), _f32p),
                                  _p(ids, _i32p), len(ids), _p(out, _f32p)) != 0:
            raise RuntimeError("oracle_pq_adc failed")
        return out

    def pq_residual_eval(self, ix, query, ids):
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        q = np.ascontiguousarray(query, dtype=np.float32)
        out = np.empty(len(ids), dtype=np.float32)
        if self.lib.oracle_pq_residual_eval(C.byref(ix[0]), _p(q, _f32p), _p(ids, _i32p), len(ids),
                                            _p(out, _f32p)) != 0:
            raise RuntimeError("oracle_pq_residual_eval failed")
        return out

    def pq_search(self, ix, graph_entry, queries, pool_sizes, entry_points, expand_count, correction=1,
                  refine_budget=0, top_k=10, threads=None, seed=42):
        queries = np.ascontiguousarray(queries, dtype=np.float32)
        nq = queries.shape[0]
        pools = np.ascontiguousarray(np.broadcast_to(np.asarray(pool_sizes, dtype=np.int32), (nq,)))
        stride = int(pools.max())
        pool_ids = np.full((nq, stride), -1, dtype=np.int32)
        pool_d = np.zeros((nq, stride), dtype=np.float32)
        pool_c = np.zeros(nq, dtype=np.int32)
        out_ids = np.full((nq, top_k), -1, dtype=np.int32)
        out_d = np.zeros((nq, top_k), dtype=np.float32)
        out_c = np.zeros(nq, dtype=np.int32)
        stats = np.zeros((nq, 4), dtype=np.uint64)
        threads = threads or min(32, os.cpu_count() or 1)
        rc = self.lib.oracle_pq_search_batch(C.byref(ix[0]), _p(queries, _f32p), nq, _p(pools, _i32p),
                                             entry_points, graph_entry, seed, expand_count, correction,
                                             refine_budget, top_k, threads, _p(pool_ids, _i32p),
                                             _p(pool_d, _f32p), stride, _p(pool_c, _i32p), _p(out_ids, _i32p),
                                             _p(out_d, _f32p), top_k, _p(out_c, _i32p), _p(stats, _u64p))
        if rc != 0:
            raise RuntimeError(f"oracle_pq_search_batch failed at query {rc - 1}")
        return dict(pool_ids=pool_ids, pool_dists=pool_d, pool_counts=pool_c, ids=out_ids, dists=out_d,
                    counts=out_c, stats=stats)

    def sq_quantize(self, ix, query):
        q = np.ascontiguousarray(query, dtype=np.float32)
        out = np.empty(ix[0].dim, dtype=np.uint8)
        self.lib.oracle_sq_quantize(C.byref(ix[0]), _p(q, _f32p), _p(out, _u8p))
        return out

    def sq_coarse(self, ix, query, ids):
        qc = self.sq_quantize(ix, query)
        return np.array([self.lib.oracle_sq_coarse(C.byref(ix[0]), _p(qc, _u8p), int(i)) for i in ids],
                        dtype=np.float32)

    def sq_exact(self, ix, query, ids):
        q = np.ascontiguousarray(query, dtype=np.float32)
        return np.array([self.lib.oracle_sq_exact(C.byref(ix[0]), _p(q, _f32p), int(i)) for i in ids],
                        dtype=np.float32)

    def sqmd_search(self, ix, graph_entry, query, pool, entry_points, expand_count, correction=1, seed=42,
                    out_cap=None):
        q = np.ascontiguousarray(query, dtype=np.float32)
        cap = out_cap or pool
        ids = np.full(cap, -1, dtype=np.int32)
        d = np.zeros(cap, dtype=np.float32)
        stats = np.zeros(4, dtype=np.uint64)
        c = self.lib.oracle_sqmd_search(C.byref(ix[0]), _p(q, _f32p), entry_points, graph_entry, seed,
                                        expand_count, pool, correction, _p(ids, _i32p), _p(d, _f32p), cap,
                                        _p(stats, _u64p))
        if c < 0:
            raise RuntimeError("oracle_sqmd_search failed")
        return ids[:c], d[:c], stats

    def dsp_search(self, ix, graph_entry, query, pool, entry_points, expand_count, num_out):
        q = np.ascontiguousarray(query, dtype=np.float32)
        ids = np.full(num_out, -1, dtype=np.int32)
        d = np.zeros(num_out, dtype=np.float32)
        c = self.lib.oracle_dsp_search(C.byref(ix[0]), _p(q, _f32p), entry_points, graph_entry, expand_count,
                                       pool, num_out, _p(ids, _i32p), _p(d, _f32p))
        if c < 0:
            raise RuntimeError("oracle_dsp_search failed")
        return ids[:c], d[:c]

    def sq_rerank(self, ix, query, ids, top_k):
        """demo_rerank_candidates restated (legacy SQ re-rank)."""
        q = np.ascontiguousarray(query, dtype=np.float32)
        work = np.array(ids, dtype=np.int32)
        wd = np.zeros(len(work), dtype=np.float32)
        out_ids = np.full(max(top_k, 1), -1, dtype=np.int32)
        out_d = np.zeros(max(top_k, 1), dtype=np.float32)
        c = self.lib.oracle_sq_rerank(C.byref(ix[0]), _p(q, _f32p), _p(work, _i32p), _p(wd, _f32p), len(work), top_k,
                                      _p(out_ids, _i32p), _p(out_d, _f32p))
        if c < 0:
            raise RuntimeError("oracle_sq_rerank failed")
        return out_ids[:c], out_d[:c]

    def refine(self, kind, ix, query, ids, top_k):
        q = np.ascontiguousarray(query, dtype=np.float32)
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        out_ids = np.full(top_k, -1, dtype=np.int32)
        out_d = np.zeros(top_k, dtype=np.float32)
        c = self.lib.oracle_refine(kind, C.cast(C.byref(ix[0]), C.c_void_p), _p(q, _f32p), _p(ids, _i32p), len(ids),
                                   top_k, _p(out_ids, _i32p), _p(out_d, _f32p))
        if c < 0:
            raise RuntimeError("oracle_refine failed")
        return out_ids[:c], out_d[:c]

    def error4(self, path, n: int, dim: int):
        """(struct, keepalive) of an ERROR4 artifact file."""
        qp, blocks, cb, vpb = read_error4(path, n, dim)
        return _Error4(_p(qp, _f32p), _p(blocks, _u8p), cb, vpb), (qp, blocks)

    def refine_ex(self, kind, ix, e4, query, ids, top_k):
        """Final refine; mode ERROR4 with e4 (from error4()), else CURRENT."""
        q = np.ascontiguousarray(query, dtype=np.float32)
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        out_ids = np.full(top_k, -1, dtype=np.int32)
        out_d = np.zeros(top_k, dtype=np.float32)
        c = self.lib.oracle_refine_ex(kind, C.cast(C.byref(ix[0]), C.c_void_p), C.byref(e4[0]) if e4 else None,
                                      _p(q, _f32p), _p(ids, _i32p), len(ids), top_k, _p(out_ids, _i32p),
                                      _p(out_d, _f32p))
        if c < 0:
            raise RuntimeError("oracle_refine_ex failed")
        return out_ids[:c], out_d[:c]

    def split_query(self, ix, query):
        sq = _SplitQuery()
        q = np.ascontiguousarray(query, dtype=np.float32)
        if self.lib.oracle_split_query(C.byref(ix[0]), _p(q, _f32p), C.byref(sq)) != 0:
            raise RuntimeError("oracle_split_query failed")
        return sq

    def split_parts(self, ix, bias, query, ids):
        """(coarse, delta, seed distance) of each id under the split distance."""
        sq = self.split_query(ix, query)
        b = np.ascontiguousarray(bias, dtype=np.float32)
        out = np.array([(self.lib.oracle_split_coarse(C.byref(ix[0]), C.byref(sq), int(i)),
                         self.lib.oracle_split_delta(C.byref(ix[0]), _p(b, _f32p), C.byref(sq), int(i)),
                         self.lib.oracle_split_distance(C.byref(ix[0]), _p(b, _f32p), C.byref(sq), int(i)))
                        for i in ids], dtype=np.float32)
        return out

    def sqmd_search_split(self, ix, bias, graph_entry, query, pool, entry_points, expand_count, seed=42,
                          out_cap=None):
        q = np.ascontiguousarray(query, dtype=np.float32)
        b = np.ascontiguousarray(bias, dtype=np.float32)
        cap = out_cap or pool
        ids = np.full(cap, -1, dtype=np.int32)
        d = np.zeros(cap, dtype=np.float32)
        stats = np.zeros(4, dtype=np.uint64)
        c = self.lib.oracle_sqmd_search_split(C.byref(ix[0]), _p(b, _f32p), _p(q, _f32p), entry_points,
                                              graph_entry, seed, expand_count, pool, _p(ids, _i32p), _p(d, _f32p),
                                              cap, _p(stats, _u64p))
        if c < 0:
            raise RuntimeError("oracle_sqmd_search_split failed")
        return ids[:c], d[:c], stats
