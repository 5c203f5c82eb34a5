"""Python binding of libcalculator.so (ctypes), the host-side mirror of the
reference's accelerator interface.

``Calculator`` exposes the reference entry points of inc/calculator.idl
(``retrieval_load`` / ``retrieval_search`` / ...) under their own names, plus
the batched extension of include/rover_b200.h.  It holds no search logic:
every call goes through the C-ABI into the CUDA library, and the library must
be present -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "lib" / "libcalculator.so"

AEE_SUCCESS = 0
AEE_EFAILED = 1
AEE_ENOMEMORY = 2
AEE_EBADPARM = 14
AEE_EUNSUPPORTED = 20

_i32p = C.POINTER(C.c_int32)
_i64p = C.POINTER(C.c_int64)
_u64p = C.POINTER(C.c_uint64)
_f32p = C.POINTER(C.c_float)
_u8p = C.POINTER(C.c_uint8)


class CalculatorError(RuntimeError):
    def __init__(self, call: str, code: int, detail: str = ""):
        super().__init__(f"{call} returned {code}" + (f": {detail}" if detail else ""))
        self.code = code


class PqIndexDesc(C.Structure):
    _fields_ = [("graph", _i32p), ("num_vectors", C.c_int32), ("graph_degree", C.c_int32),
                ("graph_entry", C.c_int32), ("dim", C.c_int32), ("codes", _u8p), ("codebook", _f32p),
                ("m", C.c_int32), ("ks", C.c_int32), ("subdim", C.c_int32), ("code_bytes", C.c_int32),
                ("residual_blocks", _u8p), ("residual_blocks_bytes", C.c_int64),
                ("residual_bits", C.c_int32), ("residual_qparams", _f32p)]


class SqIndexDesc(C.Structure):
    _fields_ = [("graph", _i32p), ("num_vectors", C.c_int32), ("graph_degree", C.c_int32),
                ("graph_entry", C.c_int32), ("dim", C.c_int32), ("l1_codes", _u8p), ("l1_bits", C.c_int32),
                ("l1_scale", C.c_float), ("l1_zero", C.c_float), ("residual_rows", _u8p),
                ("residual_bits", C.c_int32), ("residual_qparams", _f32p)]


class SearchParams(C.Structure):
    _fields_ = [("size", C.c_int32), ("mode", C.c_int32), ("entry_points", C.c_int32), ("seed", C.c_uint32),
                ("expand_count", C.c_int32), ("correction", C.c_int32), ("refine_budget", C.c_int32),
                ("top_k", C.c_int32), ("pool_stride", C.c_int32), ("sq_mode", C.c_int32),
                ("layout", C.c_int32), ("beam_width", C.c_int32), ("third_residual", C.c_int32),
                ("split_distance", C.c_int32), ("reserved", C.c_int32 * 2)]


class GateThresholds(C.Structure):
    _fields_ = [("band_lo", C.c_float), ("band_hi", C.c_float), ("refine_logit", C.c_float),
                ("stop_logit", C.c_float)]


class GateTrainParams(C.Structure):
    _fields_ = [("size", C.c_int32), ("epochs", C.c_int32), ("batch", C.c_int32), ("lr", C.c_float),
                ("beta1", C.c_float), ("beta2", C.c_float), ("eps", C.c_float), ("weight_decay", C.c_float),
                ("seed", C.c_uint32), ("pos_weight", C.c_float * 2), ("reserved", C.c_int32 * 4)]


# RoverGateTraceRow as a NumPy record (48 bytes)
TRACE_DTYPE = np.dtype([("query", np.int32), ("hop", np.int32), ("id", np.int32), ("flags", np.int32),
                        ("quantized", np.float32), ("rank", np.float32), ("worst", np.float32),
                        ("qnorm", np.float32), ("dist", np.float32), ("pad", np.float32, 3)])
GATE_PARAMS = 5 * 64 + 64 + 64 * 64 + 64 + 64 * 2 + 2
MODE_EXACT, MODE_BATCHED, MODE_GATED = 0, 1, 2


class SearchOutputs(C.Structure):
    _fields_ = [("ids", _i32p), ("dists", _f32p), ("counts", _i32p), ("out_stride", C.c_int32),
                ("pool_ids", _i32p), ("pool_dists", _f32p), ("pool_counts", _i32p), ("stats", _u64p),
                ("status", _i32p)]


class PlanInfo(C.Structure):
    _fields_ = [("num_queries", C.c_int32), ("mode", C.c_int32), ("layout", C.c_int32),
                ("warps_per_cta", C.c_int32), ("shared_visited_slots", C.c_int32), ("classes", C.c_int32),
                ("launches", C.c_int32), ("candidates", C.c_int32), ("max_pool", C.c_int32),
                ("beam_width", C.c_int32), ("class_pool", C.c_int32 * 8), ("class_queries", C.c_int32 * 8),
                ("class_blocks", C.c_int32 * 8), ("tuned_ms", C.c_float), ("default_ms", C.c_float),
                ("device_bytes", C.c_int64), ("class_split", C.c_int32), ("reserved", C.c_int32 * 7)]


class PlanConfig(C.Structure):
    _fields_ = [("layout", C.c_int32), ("warps_per_cta", C.c_int32), ("shared_visited_slots", C.c_int32),
                ("class_split", C.c_int32)]


def _p(a, t):
    return None if a is None else a.ctypes.data_as(t)


def _dp(t, ptr):
    """A raw device pointer (int) as a ctypes pointer."""
    return C.cast(C.c_void_p(int(ptr)), t) if ptr else None


def load_library(path: str | Path | None = None) -> C.CDLL:
    path = Path(path or LIB_PATH)
    if not path.is_file():
        raise FileNotFoundError(f"{path} is missing: build it with `python -m rover_b200.build`")
    return C.CDLL(str(path))


class Calculator:
    """One session handle on the process-wide device state."""

    def __init__(self, lib_path: str | Path | None = None):
        self.lib = load_library(lib_path)
        L = self.lib
        L.calculator_open.argtypes = [C.c_char_p, C.POINTER(C.c_uint64)]
        L.calculator_close.argtypes = [C.c_uint64]
        L.calculator_rover_configure.argtypes = [C.c_uint64, C.c_int32, C.c_int32]
        L.calculator_retrieval_load.argtypes = [C.c_uint64, _i32p, C.c_int, _u8p, C.c_int, C.c_int32, C.c_int32,
                                                C.c_int32, C.c_int32, C.c_float, C.c_float]
        L.calculator_retrieval_search.argtypes = [C.c_uint64, _f32p, C.c_int, C.c_int32, C.c_int32, C.c_int32,
                                                  C.c_int32, _i32p, C.c_int, _f32p, C.c_int, _i32p]
        L.calculator_retrieval_unload.argtypes = [C.c_uint64]
        L.calculator_rover_last_error.restype = C.c_char_p
        L.calculator_rover_launch_count.restype = C.c_uint64
        L.calculator_rover_gate_load.argtypes = [C.c_uint64, _f32p, _f32p, _f32p, C.POINTER(GateThresholds)]
        L.calculator_rover_gate_unload.argtypes = [C.c_uint64]
        L.calculator_rover_gate_rows.argtypes = [C.c_uint64, C.POINTER(C.c_uint64)]
        L.calculator_rover_seed_rank.argtypes = [C.c_uint64, _f32p, C.c_int32, _f32p, C.c_int32, C.c_int32, _f32p]
        L.calculator_rover_gate_eval.argtypes = [C.c_uint64, _f32p, C.c_int64, _f32p]
        L.calculator_rover_seed_topm.argtypes = [C.c_uint64, _f32p, C.c_int32, C.c_int32, C.c_int32, _u64p, _f32p]
        L.calculator_rover_gate_train.argtypes = [C.c_uint64, _f32p, _f32p, _f32p, C.c_int64,
                                                  C.POINTER(GateTrainParams), _f32p, _f32p, _f32p, _f32p]
        L.calculator_rover_gate_grad.argtypes = [C.c_uint64, _f32p, _f32p, _f32p, C.c_int64, _f32p, _f32p, _f32p,
                                                 _f32p, _f32p, _f32p]
        L.calculator_rover_pq_trace.argtypes = [C.c_uint64, C.POINTER(SearchParams), _f32p, C.c_int32, _i32p,
                                                C.POINTER(SearchOutputs), C.c_void_p, C.c_int64, _i64p]
        L.calculator_rover_kernel_timing.argtypes = [C.c_int32]
        L.calculator_rover_kernel_times.argtypes = [_i64p, C.POINTER(C.c_double), C.c_int32]
        L.calculator_rover_kernel_times.restype = C.c_int32
        L.calculator_rover_pq_load.argtypes = [C.c_uint64, C.POINTER(PqIndexDesc)]
        L.calculator_rover_pq_unload.argtypes = [C.c_uint64]
        L.calculator_rover_pq_search.argtypes = [C.c_uint64, C.POINTER(SearchParams), _f32p, C.c_int32, _i32p,
                                                 _i32p, C.POINTER(SearchOutputs)]
        L.calculator_rover_pq_search_device.argtypes = [C.c_uint64, C.POINTER(SearchParams), _f32p, C.c_int32,
                                                        _i32p, _i32p, C.POINTER(SearchOutputs), C.c_void_p]
        L.calculator_rover_pq_plan_create.argtypes = [C.c_uint64, C.POINTER(SearchParams), C.c_int32, _i32p, _i32p,
                                                      _f32p, C.POINTER(C.c_void_p)]
        L.calculator_rover_pq_plan_create_fixed.argtypes = [C.c_uint64, C.POINTER(SearchParams), C.c_int32, _i32p,
                                                            _i32p, C.POINTER(PlanConfig), C.POINTER(C.c_void_p)]
        L.calculator_rover_pq_plan_launch.argtypes = [C.c_void_p, _f32p, C.POINTER(SearchOutputs), C.c_void_p]
        L.calculator_rover_pq_plan_describe.argtypes = [C.c_void_p, C.POINTER(PlanInfo)]
        L.calculator_rover_pq_plan_destroy.argtypes = [C.c_void_p]
        L.calculator_rover_score.argtypes = [C.c_uint64, C.c_int32, _f32p, C.c_int32, _i32p, _i64p, _f32p, _i32p]
        L.calculator_rover_pq_lut.argtypes = [C.c_uint64, _f32p, C.c_int32, _f32p, _i32p]
        L.calculator_rover_refine.argtypes = [C.c_uint64, C.c_int32, _f32p, C.c_int32, _i32p, C.c_int32, _i32p,
                                              C.c_int32, _i32p, _f32p, _i32p, _i32p]
        L.calculator_rover_sq_load.argtypes = [C.c_uint64, C.POINTER(SqIndexDesc)]
        L.calculator_rover_sq_unload.argtypes = [C.c_uint64]
        L.calculator_rover_sq_search.argtypes = [C.c_uint64, C.POINTER(SearchParams), _f32p, C.c_int32, _i32p,
                                                 C.POINTER(SearchOutputs)]
        L.calculator_rover_error4_load.argtypes = [C.c_uint64, C.c_int32, _f32p, _u8p, C.c_int64, C.c_int32,
                                                   C.c_int32]
        L.calculator_rover_error4_unload.argtypes = [C.c_uint64, C.c_int32]
        L.calculator_rover_sq_split_load.argtypes = [C.c_uint64, _f32p, C.c_int32]
        L.calculator_rover_pq_train.argtypes = [C.c_uint64, _f32p, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                                C.c_int32, _f32p]
        L.calculator_rover_pq_encode.argtypes = [C.c_uint64, _f32p, C.c_int64, C.c_int32, _f32p, C.c_int32,
                                                 C.c_int32, _u8p]
        self.handle = C.c_uint64(0)
        self._check("calculator_open", L.calculator_open(b"file:///libcalculator_skel.so", C.byref(self.handle)))
        self._keep = {}

    # -- helpers
    def last_error(self) -> str:
        return (self.lib.calculator_rover_last_error() or b"").decode()

    def _check(self, call, rc):
        if rc != AEE_SUCCESS:
            raise CalculatorError(call, rc, self.last_error())
        return rc

    def launch_count(self) -> int:
        return int(self.lib.calculator_rover_launch_count())

    KERNEL_KINDS = ("pq_packed", "pq_seeds", "pq_decoded", "pq_batched", "sq", "pq_seed_rank", "pq_lut", "pq_adc",
                    "pq_residual", "sq_coarse", "sq_exact", "refine", "pq_rescore", "plan", "pq_seed_topm",
                    "pq_train")

    # -- learned gate
    def gate_load(self, params, mu, sigma, band_lo=0.0, band_hi=0.0, refine_logit=0.0, stop_logit=1e30) -> None:
        p = np.ascontiguousarray(params, np.float32)
        m = np.ascontiguousarray(mu, np.float32)
        sg = np.ascontiguousarray(sigma, np.float32)
        t = GateThresholds(band_lo, band_hi, refine_logit, stop_logit)
        self._check("calculator_rover_gate_load",
                    self.lib.calculator_rover_gate_load(self.handle, _p(p, _f32p), _p(m, _f32p), _p(sg, _f32p),
                                                        C.byref(t)))

    def seed_rank(self, queries, rows) -> np.ndarray:
        """[nq][n_rows] TF32 tensor-core ranks |q|^2 + |x|^2 - 2 q.x (clamped at 0)."""
        q = np.ascontiguousarray(queries, dtype=np.float32)
        x = np.ascontiguousarray(rows, dtype=np.float32)
        out = np.empty((q.shape[0], x.shape[0]), np.float32)
        self._check("calculator_rover_seed_rank",
                    self.lib.calculator_rover_seed_rank(self.handle, _p(q, _f32p), q.shape[0], _p(x, _f32p),
                                                        x.shape[0], q.shape[1], _p(out, _f32p)))
        return out

    def gate_rows(self) -> int:
        """MLP rows the loaded gate has evaluated inside searches since it was loaded."""
        v = C.c_uint64()
        self._check("calculator_rover_gate_rows", self.lib.calculator_rover_gate_rows(self.handle, C.byref(v)))
        return int(v.value)

    def gate_unload(self) -> None:
        self._check("calculator_rover_gate_unload", self.lib.calculator_rover_gate_unload(self.handle))

    def gate_eval(self, rows) -> np.ndarray:
        """The loaded gate's logits [n][2] for raw rows [n][5] (quantized
        distance, rank / L, worst distance, hop / L, query norm)."""
        x = np.ascontiguousarray(rows, dtype=np.float32).reshape(-1, 5)
        out = np.zeros((len(x), 2), np.float32)
        self._check("calculator_rover_gate_eval",
                    self.lib.calculator_rover_gate_eval(self.handle, _p(x, _f32p), len(x), _p(out, _f32p)))
        return out

    def seed_topm(self, rank, m: int):
        """The m smallest (rank bits << 32 | seed index) keys of each row of
        rank [rows][n_seeds] ascending, and each row's (m+1)-th rank, as the
        verified seed pool selects them on the device."""
        r = np.ascontiguousarray(rank, dtype=np.float32)
        rows, n = r.shape
        keys = np.zeros((rows, m), np.uint64)
        nxt = np.zeros(rows, np.float32)
        self._check("calculator_rover_seed_topm",
                    self.lib.calculator_rover_seed_topm(self.handle, _p(r, _f32p), rows, n, m, _p(keys, _u64p),
                                                        _p(nxt, _f32p)))
        return keys, nxt

    def gate_train(self, x, y, m, epochs=4, batch=4096, lr=2e-3, weight_decay=0.0, seed=1,
                   pos_weight=(1.0, 1.0)) -> dict:
        """Trains the gate on the device; returns params, mu, sigma, losses."""
        x = np.ascontiguousarray(x, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        m = np.ascontiguousarray(m, np.float32)
        n = x.shape[0]
        tp = GateTrainParams()
        tp.size = C.sizeof(GateTrainParams)
        tp.epochs, tp.batch, tp.lr = epochs, batch, lr
        tp.beta1, tp.beta2, tp.eps, tp.weight_decay, tp.seed = 0.9, 0.999, 1e-8, weight_decay, seed
        tp.pos_weight[0], tp.pos_weight[1] = pos_weight
        params = np.zeros(GATE_PARAMS, np.float32)
        mu = np.zeros(5, np.float32)
        sigma = np.zeros(5, np.float32)
        losses = np.zeros(epochs, np.float32)
        self._check("calculator_rover_gate_train",
                    self.lib.calculator_rover_gate_train(self.handle, _p(x, _f32p), _p(y, _f32p), _p(m, _f32p), n,
                                                         C.byref(tp), _p(params, _f32p), _p(mu, _f32p),
                                                         _p(sigma, _f32p), _p(losses, _f32p)))
        return dict(params=params, mu=mu, sigma=sigma, losses=losses)

    def gate_grad(self, x, y, m, params, mu, sigma, pos_weight=(1.0, 1.0)):
        x = np.ascontiguousarray(x, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        m = np.ascontiguousarray(m, np.float32)
        p = np.ascontiguousarray(params, np.float32)
        mu = np.ascontiguousarray(mu, np.float32)
        sg = np.ascontiguousarray(sigma, np.float32)
        pw = np.ascontiguousarray(pos_weight, np.float32)
        grad = np.zeros(GATE_PARAMS, np.float32)
        loss = np.zeros(1, np.float32)
        self._check("calculator_rover_gate_grad",
                    self.lib.calculator_rover_gate_grad(self.handle, _p(x, _f32p), _p(y, _f32p), _p(m, _f32p),
                                                        x.shape[0], _p(p, _f32p), _p(mu, _f32p), _p(sg, _f32p),
                                                        _p(pw, _f32p), _p(grad, _f32p), _p(loss, _f32p)))
        return float(loss[0]), grad

    def pq_trace(self, queries, pool_sizes, capacity, top_k=10, **kw) -> dict:
        """Plain search with full correction in the reference's order,
        returning its results and the gate's trace rows."""
        q = np.ascontiguousarray(queries, dtype=np.float32)
        nq = q.shape[0]
        pools = np.ascontiguousarray(np.broadcast_to(np.asarray(pool_sizes, dtype=np.int32), (nq,)))
        p = self.params(top_k=top_k, **kw)
        r = dict(ids=np.full((nq, top_k), -1, np.int32), dists=np.zeros((nq, top_k), np.float32),
                 counts=np.zeros(nq, np.int32), status=np.zeros(nq, np.int32), stats=np.zeros((nq, 4), np.uint64))
        o = SearchOutputs(_p(r["ids"], _i32p), _p(r["dists"], _f32p), _p(r["counts"], _i32p), top_k, None, None,
                          None, _p(r["stats"], _u64p), _p(r["status"], _i32p))
        rows = np.zeros(int(capacity), TRACE_DTYPE)
        count = C.c_int64(0)
        self._check("calculator_rover_pq_trace",
                    self.lib.calculator_rover_pq_trace(self.handle, C.byref(p), _p(q, _f32p), nq, _p(pools, _i32p),
                                                       C.byref(o), rows.ctypes.data_as(C.c_void_p), int(capacity),
                                                       C.byref(count)))
        r["rows"] = rows[:min(int(capacity), count.value)]
        r["row_count"] = count.value
        return r

    def kernel_timing(self, enable: bool = True) -> None:
        """Turn per-kernel event timing on or off (and reset the totals)."""
        self.lib.calculator_rover_kernel_timing(1 if enable else 0)

    def kernel_times(self) -> dict:
        """{kind: (launches, total ms)} since the last kernel_timing call."""
        n = 16
        launches = np.zeros(n, np.int64)
        ms = np.zeros(n, np.float64)
        self.lib.calculator_rover_kernel_times(_p(launches, _i64p), ms.ctypes.data_as(C.POINTER(C.c_double)), n)
        return {k: (int(launches[i]), float(ms[i])) for i, k in enumerate(self.KERNEL_KINDS)}

    def close(self):
        if self.handle.value:
            self.lib.calculator_close(self.handle)
            self.handle = C.c_uint64(0)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- reference entry points (calculator.idl)
    def rover_configure(self, abi_version: int, l1_bits: int) -> int:
        return self.lib.calculator_rover_configure(self.handle, abi_version, l1_bits)

    def retrieval_load(self, graph, l1_codes, num_vectors, dim, graph_k, graph_entry, l1_scale, l1_zero) -> int:
        g = np.ascontiguousarray(graph, dtype=np.int32).reshape(-1)
        c = np.ascontiguousarray(l1_codes, dtype=np.uint8).reshape(-1)
        return self.lib.calculator_retrieval_load(self.handle, _p(g, _i32p), g.size, _p(c, _u8p), c.size,
                                                  num_vectors, dim, graph_k, graph_entry, l1_scale, l1_zero)

    def retrieval_search(self, query, entry_points, expand_count, pool_size, num_out):
        q = np.ascontiguousarray(query, dtype=np.float32)
        ids = np.full(num_out, -1, dtype=np.int32)
        d = np.zeros(num_out, dtype=np.float32)
        actual = C.c_int32(0)
        rc = self.lib.calculator_retrieval_search(self.handle, _p(q, _f32p), q.size, entry_points, expand_count,
                                                  pool_size, num_out, _p(ids, _i32p), num_out, _p(d, _f32p),
                                                  num_out, C.byref(actual))
        return rc, ids[:actual.value], d[:actual.value]

    def retrieval_unload(self) -> int:
        return self.lib.calculator_retrieval_unload(self.handle)

    # -- extension: PQ
    def pq_load(self, graph, graph_entry: int, bundle) -> None:
        """graph: [n][degree] int32 or None; bundle: rover_b200.bundle.PqBundle."""
        md = bundle.meta
        g = None if graph is None else np.ascontiguousarray(graph, dtype=np.int32)
        codes = np.ascontiguousarray(bundle.codes, dtype=np.uint8)
        book = np.ascontiguousarray(bundle.codebook, dtype=np.float32)
        res = np.ascontiguousarray(bundle.residual_blocks, dtype=np.uint8) if bundle.residual_bits else None
        qp = np.ascontiguousarray(bundle.qparams, dtype=np.float32) if bundle.residual_bits else None
        desc = PqIndexDesc(_p(g, _i32p), md.num_vectors, 0 if g is None else g.shape[1], graph_entry, md.dim,
                           _p(codes, _u8p), _p(book, _f32p), md.m, md.ks, md.subdim, md.code_bytes,
                           _p(res, _u8p), 0 if res is None else res.size, bundle.residual_bits, _p(qp, _f32p))
        self._check("calculator_rover_pq_load", self.lib.calculator_rover_pq_load(self.handle, C.byref(desc)))
        self.pq_dim = md.dim

    def pq_unload(self):
        self.lib.calculator_rover_pq_unload(self.handle)

    @staticmethod
    def params(entry_points=1, expand_count=32, correction=1, refine_budget=0, top_k=10, seed=42,
               pool_stride=0, sq_mode=0, mode=0, layout=0, beam_width=0, third_residual=0,
               split_distance=0) -> SearchParams:
        p = SearchParams()
        p.size = C.sizeof(SearchParams)
        p.mode = mode
        p.entry_points = entry_points
        p.seed = seed
        p.expand_count = expand_count
        p.correction = correction
        p.refine_budget = refine_budget
        p.top_k = top_k
        p.pool_stride = pool_stride
        p.sq_mode = sq_mode
        p.layout = layout
        p.beam_width = beam_width
        p.third_residual = third_residual
        p.split_distance = split_distance
        return p

    def pq_search(self, queries, pool_sizes, top_k=10, top_ks=None, pool_stride=0, stats=True, check=True,
                  out: dict | None = None, **kw) -> dict:
        """Host-buffer search (calculator_rover_pq_search).  out: arrays from
        an earlier call's result to write into again (ids, dists, counts,
        status of the same shapes), so that repeated calls allocate nothing;
        the call fills every row it returns (counts give the valid prefix)."""
        q = np.ascontiguousarray(queries, dtype=np.float32)
        nq = q.shape[0]
        pools = np.ascontiguousarray(np.broadcast_to(np.asarray(pool_sizes, dtype=np.int32), (nq,)))
        tks = None if top_ks is None else np.ascontiguousarray(np.broadcast_to(np.asarray(top_ks, dtype=np.int32), (nq,)))
        stride = top_k if tks is None else int(tks.max())
        p = self.params(top_k=top_k, pool_stride=pool_stride, **kw)
        if out is not None and not pool_stride and not stats and out["ids"].shape == (nq, stride):
            r = {k: out[k] for k in ("ids", "dists", "counts", "status")}
        else:
            r = dict(ids=np.full((nq, stride), -1, np.int32), dists=np.zeros((nq, stride), np.float32),
                     counts=np.zeros(nq, np.int32), status=np.zeros(nq, np.int32))
        if pool_stride:
            r.update(pool_ids=np.full((nq, pool_stride), -1, np.int32),
                     pool_dists=np.zeros((nq, pool_stride), np.float32), pool_counts=np.zeros(nq, np.int32))
        if stats:
            r["stats"] = np.zeros((nq, 4), np.uint64)
        o = SearchOutputs(_p(r["ids"], _i32p), _p(r["dists"], _f32p), _p(r["counts"], _i32p), stride,
                          _p(r.get("pool_ids"), _i32p), _p(r.get("pool_dists"), _f32p),
                          _p(r.get("pool_counts"), _i32p), _p(r.get("stats"), _u64p), _p(r["status"], _i32p))
        rc = self.lib.calculator_rover_pq_search(self.handle, C.byref(p), _p(q, _f32p), nq, _p(pools, _i32p),
                                                 _p(tks, _i32p), C.byref(o))
        r["rc"] = rc
        if check:
            self._check("calculator_rover_pq_search", rc)
        return r

    def pq_search_device(self, queries_ptr: int, nq: int, pool_ptr: int, out: dict, topk_ptr: int = 0,
                         stream_ptr: int = 0, check=True, **kw) -> int:
        """Device-resident variant: pointers are raw CUDA device addresses
        (e.g. torch tensor .data_ptr()).  out holds device pointers for the
        keys ids, dists, counts, stride and optionally pool_*, stats, status."""
        p = self.params(**kw)
        o = SearchOutputs(_dp(_i32p, out.get("ids")), _dp(_f32p, out.get("dists")), _dp(_i32p, out.get("counts")),
                          out.get("stride", 0), _dp(_i32p, out.get("pool_ids")), _dp(_f32p, out.get("pool_dists")),
                          _dp(_i32p, out.get("pool_counts")), _dp(_u64p, out.get("stats")),
                          _dp(_i32p, out.get("status")))
        rc = self.lib.calculator_rover_pq_search_device(self.handle, C.byref(p), _dp(_f32p, queries_ptr), nq,
                                                        _dp(_i32p, pool_ptr), _dp(_i32p, topk_ptr), C.byref(o),
                                                        C.c_void_p(stream_ptr or None))
        if check:
            self._check("calculator_rover_pq_search_device", rc)
        return rc

    def pq_plan(self, nq: int, pool_sizes, top_ks=None, tune_queries_ptr: int = 0, top_k: int = 10,
                config=None, **kw) -> "Plan":
        """A search plan (calculator_rover_pq_plan_create) for nq queries with
        these beam widths and result counts.  tune_queries_ptr: device address
        of [nq][dim] FP32 queries to tune on (0 = no tuning).  config (a dict
        with the keys of describe(), or a (layout, warps_per_cta,
        shared_visited_slots, class_split) tuple) pins a configuration
        instead (calculator_rover_pq_plan_create_fixed)."""
        pools = np.ascontiguousarray(np.broadcast_to(np.asarray(pool_sizes, dtype=np.int32), (nq,)))
        tks = None if top_ks is None else np.ascontiguousarray(np.broadcast_to(np.asarray(top_ks, dtype=np.int32), (nq,)))
        p = self.params(top_k=top_k, **kw)
        h = C.c_void_p()
        if config is not None:
            cfg = PlanConfig(*config) if not isinstance(config, dict) else PlanConfig(
                config["layout"], config["warps_per_cta"], config["shared_visited_slots"], config["class_split"])
            rc = self.lib.calculator_rover_pq_plan_create_fixed(self.handle, C.byref(p), nq, _p(pools, _i32p),
                                                                _p(tks, _i32p), C.byref(cfg), C.byref(h))
            self._check("calculator_rover_pq_plan_create_fixed", rc)
        else:
            rc = self.lib.calculator_rover_pq_plan_create(self.handle, C.byref(p), nq, _p(pools, _i32p),
                                                          _p(tks, _i32p), _dp(_f32p, tune_queries_ptr), C.byref(h))
            self._check("calculator_rover_pq_plan_create", rc)
        return Plan(self, h, nq, int(tks.max()) if tks is not None else top_k)

    def pq_lut(self, queries, m, ks):
        q = np.ascontiguousarray(queries, dtype=np.float32)
        out = np.zeros((q.shape[0], m * ks), np.float32)
        st = np.zeros(q.shape[0], np.int32)
        self._check("calculator_rover_pq_lut",
                    self.lib.calculator_rover_pq_lut(self.handle, _p(q, _f32p), q.shape[0], _p(out, _f32p),
                                                     _p(st, _i32p)))
        return out

    def score(self, kind: int, queries, id_lists):
        q = np.ascontiguousarray(queries, dtype=np.float32)
        offsets = np.zeros(len(id_lists) + 1, np.int64)
        offsets[1:] = np.cumsum([len(x) for x in id_lists])
        ids = np.ascontiguousarray(np.concatenate([np.asarray(x, np.int32) for x in id_lists])
                                   if len(id_lists) else np.zeros(0, np.int32), dtype=np.int32)
        out = np.zeros(max(1, int(offsets[-1])), np.float32)
        st = np.zeros(q.shape[0], np.int32)
        self._check("calculator_rover_score",
                    self.lib.calculator_rover_score(self.handle, kind, _p(q, _f32p), q.shape[0], _p(ids, _i32p),
                                                    _p(offsets, _i64p), _p(out, _f32p), _p(st, _i32p)))
        return [out[offsets[i]:offsets[i + 1]] for i in range(len(id_lists))]

    def refine(self, kind, queries, cand_ids, cand_counts, top_k):
        q = np.ascontiguousarray(queries, dtype=np.float32)
        ids = np.ascontiguousarray(cand_ids, dtype=np.int32)
        counts = np.ascontiguousarray(cand_counts, dtype=np.int32)
        nq = q.shape[0]
        oi = np.full((nq, top_k), -1, np.int32)
        od = np.zeros((nq, top_k), np.float32)
        oc = np.zeros(nq, np.int32)
        st = np.zeros(nq, np.int32)
        self._check("calculator_rover_refine",
                    self.lib.calculator_rover_refine(self.handle, kind, _p(q, _f32p), nq, _p(ids, _i32p),
                                                     ids.shape[1], _p(counts, _i32p), top_k, _p(oi, _i32p),
                                                     _p(od, _f32p), _p(oc, _i32p), _p(st, _i32p)))
        return oi, od, oc

    def pq_train(self, vectors, m: int, ks: int, iters: int) -> np.ndarray:
        """retrieval_pq_train on the GPU: codebook [m][ks][dim/m]."""
        x = np.ascontiguousarray(vectors, dtype=np.float32)
        n, dim = x.shape
        book = np.zeros((m, ks, dim // m), np.float32)
        self._check("calculator_rover_pq_train",
                    self.lib.calculator_rover_pq_train(self.handle, _p(x, _f32p), n, dim, m, ks, iters,
                                                       _p(book, _f32p)))
        return book

    def pq_encode(self, vectors, codebook) -> np.ndarray:
        """retrieval_pq_encode_batch on the GPU: codes [n][code_bytes]."""
        x = np.ascontiguousarray(vectors, dtype=np.float32)
        book = np.ascontiguousarray(codebook, dtype=np.float32)
        m, ks, _ = book.shape
        cb = (m + 1) // 2 if ks <= 16 else m
        codes = np.zeros((x.shape[0], cb), np.uint8)
        self._check("calculator_rover_pq_encode",
                    self.lib.calculator_rover_pq_encode(self.handle, _p(x, _f32p), x.shape[0], x.shape[1],
                                                        _p(book, _f32p), m, ks, _p(codes, _u8p)))
        return codes

    def error4_load(self, kind: int, qparams, code_blocks) -> None:
        """The ERROR4 artifact payload (qparams [n][2], 4096-byte code blocks)
        of the loaded SQ (kind 0) or PQ (kind 1) index."""
        qp = np.ascontiguousarray(qparams, dtype=np.float32)
        blocks = np.ascontiguousarray(code_blocks, dtype=np.uint8).reshape(-1)
        dim = self.pq_dim if kind == 1 else self._keep["sq_dim"]
        self._check("calculator_rover_error4_load",
                    self.lib.calculator_rover_error4_load(self.handle, kind, _p(qp, _f32p), _p(blocks, _u8p),
                                                          blocks.size, qp.shape[0], dim))

    def error4_unload(self, kind: int) -> None:
        self._check("calculator_rover_error4_unload", self.lib.calculator_rover_error4_unload(self.handle, kind))

    def sq_split_load(self, bias) -> None:
        """The SQ4 split-distance bias of the loaded SQ index."""
        b = np.ascontiguousarray(bias, dtype=np.float32)
        self._check("calculator_rover_sq_split_load",
                    self.lib.calculator_rover_sq_split_load(self.handle, _p(b, _f32p), b.size))

    # -- extension: SQ
    def sq_load(self, graph, graph_entry: int, b) -> None:
        g = None if graph is None else np.ascontiguousarray(graph, dtype=np.int32)
        l1 = np.ascontiguousarray(b.l1, dtype=np.uint8)
        res = np.ascontiguousarray(b.residual_rows, dtype=np.uint8)
        qp = np.ascontiguousarray(b.qparams, dtype=np.float32)
        self._keep["sq"] = (g, l1, res, qp)
        desc = SqIndexDesc(_p(g, _i32p), b.num_vectors, 0 if g is None else g.shape[1], graph_entry, b.dim,
                           _p(l1, _u8p), b.l1_bits, b.l1_scale, b.l1_zero, _p(res, _u8p), b.residual_bits,
                           _p(qp, _f32p))
        self._check("calculator_rover_sq_load", self.lib.calculator_rover_sq_load(self.handle, C.byref(desc)))
        self._keep["sq_dim"] = b.dim

    def sq_unload(self) -> None:
        self._check("calculator_rover_sq_unload", self.lib.calculator_rover_sq_unload(self.handle))
        self._keep.pop("sq", None)

    def sq_search(self, queries, pool_sizes, out_stride, sq_mode=1, num_out=None, check=True, **kw) -> dict:
        q = np.ascontiguousarray(queries, dtype=np.float32)
        nq = q.shape[0]
        pools = np.ascontiguousarray(np.broadcast_to(np.asarray(pool_sizes, dtype=np.int32), (nq,)))
        p = self.params(sq_mode=sq_mode, top_k=num_out or out_stride, **kw)
        r = dict(ids=np.full((nq, out_stride), -1, np.int32), dists=np.zeros((nq, out_stride), np.float32),
                 counts=np.zeros(nq, np.int32), status=np.zeros(nq, np.int32), stats=np.zeros((nq, 4), np.uint64))
        o = SearchOutputs(_p(r["ids"], _i32p), _p(r["dists"], _f32p), _p(r["counts"], _i32p), out_stride,
                          None, None, None, _p(r["stats"], _u64p), _p(r["status"], _i32p))
        rc = self.lib.calculator_rover_sq_search(self.handle, C.byref(p), _p(q, _f32p), nq, _p(pools, _i32p),
                                                 C.byref(o))
        r["rc"] = rc
        if check:
            self._check("calculator_rover_sq_search", rc)
        return r


class Plan:
    """A search plan: the same searches enqueued on new query vectors.  Every
    pointer is a raw CUDA device address (e.g. torch tensor .data_ptr())."""

    def __init__(self, calc: Calculator, handle: C.c_void_p, nq: int, max_k: int):
        self.calc = calc
        self.handle = handle
        self.nq = nq
        self.max_k = max_k

    def launch(self, queries_ptr: int, out: dict, stream_ptr: int = 0) -> None:
        """Enqueue (no wait).  out holds device pointers for ids, dists, counts,
        stride, status (required) and optionally pool_*, stats."""
        o = SearchOutputs(_dp(_i32p, out.get("ids")), _dp(_f32p, out.get("dists")), _dp(_i32p, out.get("counts")),
                          out.get("stride", 0), _dp(_i32p, out.get("pool_ids")), _dp(_f32p, out.get("pool_dists")),
                          _dp(_i32p, out.get("pool_counts")), _dp(_u64p, out.get("stats")),
                          _dp(_i32p, out.get("status")))
        rc = self.calc.lib.calculator_rover_pq_plan_launch(self.handle, _dp(_f32p, queries_ptr), C.byref(o),
                                                           C.c_void_p(stream_ptr or None))
        self.calc._check("calculator_rover_pq_plan_launch", rc)

    def describe(self) -> dict:
        info = PlanInfo()
        self.calc._check("calculator_rover_pq_plan_describe",
                         self.calc.lib.calculator_rover_pq_plan_describe(self.handle, C.byref(info)))
        n = info.classes
        return dict(num_queries=info.num_queries, mode=info.mode, layout=info.layout,
                    warps_per_cta=info.warps_per_cta, shared_visited_slots=info.shared_visited_slots,
                    classes=n, launches=info.launches, candidates=info.candidates, max_pool=info.max_pool,
                    beam_width=info.beam_width, class_pool=list(info.class_pool[:n]),
                    class_queries=list(info.class_queries[:n]), class_blocks=list(info.class_blocks[:n]),
                    tuned_ms=info.tuned_ms, default_ms=info.default_ms, device_bytes=info.device_bytes,
                    class_split=info.class_split)

    def destroy(self) -> None:
        if self.handle:
            self.calc.lib.calculator_rover_pq_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass
