"""Neighbourhood-aware id layout of a PQ index (the reference's rover-layout
tool, src/graph/layout_opt_kmeans.cpp): the ordering itself runs in C++ in
librover_host.so (rover_layout_order); this module binds it and applies an
order to a workload, the way the reference's `gorder` bundles carry it
(tools/index_bundle.py: the graph, codes, residual rows and qparams stored
in the new order, with an order map new id -> original id)."""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import replace

import numpy as np

from . import bundle as B
from .build import HOST_LIB


def _lib():
    lib = C.CDLL(str(HOST_LIB))
    p32 = C.POINTER(C.c_int32)
    lib.rover_layout_order.argtypes = [p32, C.c_int32, C.c_int32, p32, C.c_int32, C.c_int32, C.c_double,
                                       C.c_int32, C.c_int32, C.c_int32, C.c_int32, p32]
    return lib


def gorder(graph: np.ndarray, labels: np.ndarray, clusters: int, vectors_per_block: int, rrf_c: float = 60.0,
           max_reverse: int = 1024, use_cn: bool = True, use_mnn: bool = True, threads: int | None = None):
    """new_to_old order of the graph's ids (new id -> old id)."""
    g = np.ascontiguousarray(graph, dtype=np.int32)
    lab = np.ascontiguousarray(labels, dtype=np.int32)
    out = np.empty(g.shape[0], dtype=np.int32)
    p32 = C.POINTER(C.c_int32)
    rc = _lib().rover_layout_order(g.ctypes.data_as(p32), g.shape[0], g.shape[1], lab.ctypes.data_as(p32),
                                   clusters, vectors_per_block, rrf_c, max_reverse, int(use_cn), int(use_mnn),
                                   threads or os.cpu_count() or 1, out.ctypes.data_as(p32))
    if rc != 0:
        raise ValueError("rover_layout_order rejected its input")
    return out


def permute_pq(w, new_to_old: np.ndarray):
    """The workload w (workloads.PqWorkload) with its ids in the new order:
    graph rows and entries renumbered, codes / residual rows / qparams moved,
    ground truth renumbered.  Returns (workload, new_to_old)."""
    n2o = np.asarray(new_to_old, dtype=np.int64)
    o2n = np.empty_like(n2o)
    o2n[n2o] = np.arange(len(n2o))
    g = w.graph[n2o]
    graph = np.where(g >= 0, o2n[np.maximum(g, 0)], -1).astype(np.int32)
    b = w.bundle
    rows = b.residual_rows()[n2o]
    bundle = B.PqBundle(b.meta, b.codebook, np.ascontiguousarray(b.codes[n2o]), b.residual_bits,
                        B.pack_residual_blocks(rows), np.ascontiguousarray(b.qparams[n2o]))
    gt = np.where(w.gt >= 0, o2n[np.maximum(w.gt, 0)], -1).astype(np.int32)
    return replace(w, graph=graph, entry=int(o2n[w.entry]), bundle=bundle, gt=gt), new_to_old


def nearest_centre(base: np.ndarray, centers: np.ndarray) -> np.ndarray:
    """Index of each vector's nearest centre (squared L2; torch, on the GPU
    when there is one), 65,536 vectors at a time."""
    import torch
    dev = torch.device("cuda" if torch.cuda.is_available() else "cpu")
    with torch.no_grad():
        c = torch.from_numpy(np.ascontiguousarray(centers, dtype=np.float32)).to(dev)
        cn = (c * c).sum(1)
        parts = []
        for s in range(0, base.shape[0], 65536):
            x = torch.from_numpy(np.ascontiguousarray(base[s:s + 65536], dtype=np.float32)).to(dev)
            parts.append(torch.argmin(cn[None, :] - 2.0 * (x @ c.T), dim=1).int().cpu())
        return torch.cat(parts).numpy()


def gorder_workload(w, per_block: int = 32, threads: int | None = None):
    """The workload's layout by gorder, clustered by the nearest mixture
    centre (the mixture the workload was drawn from; rover_b200.workloads
    CONFIGS).  Returns (workload, new_to_old)."""
    from . import datasets as D
    from .workloads import CONFIGS
    cfg = CONFIGS[w.name]
    base, centers = D.gmm(cfg["n"], cfg["dim"], cfg["comps"], cfg["seed"], clip_nonneg=cfg["clip"],
                          normalize=cfg["normalize"], return_centers=True)
    labels = nearest_centre(base, centers)
    n2o = gorder(w.graph, labels, int(centers.shape[0]), per_block, threads=threads)
    return permute_pq(w, n2o)


def permute_large(w, new_to_old: np.ndarray):
    """The large combined workload (workloads.LargeWorkload) with its ids in
    the new order: graph renumbered, the PQ bundle's and the SQ bundle's rows
    moved, ground truth and entry renumbered.  Returns (workload,
    new_to_old)."""
    n2o = np.asarray(new_to_old, dtype=np.int64)
    o2n = np.empty_like(n2o)
    o2n[n2o] = np.arange(len(n2o))
    g = w.graph[n2o]
    graph = np.where(g >= 0, o2n[np.maximum(g, 0)], -1).astype(np.int32)
    del g
    p = w.pq
    pq = B.PqBundle(p.meta, p.codebook, np.ascontiguousarray(p.codes[n2o]), p.residual_bits,
                    B.pack_residual_blocks(p.residual_rows()[n2o]), np.ascontiguousarray(p.qparams[n2o]))
    q = w.sq
    sq = B.SqBundle(q.num_vectors, q.dim, q.l1_bits, q.l1_scale, q.l1_zero, np.ascontiguousarray(q.l1[n2o]),
                    q.residual_bits, np.ascontiguousarray(q.residual_rows[n2o]), np.ascontiguousarray(q.qparams[n2o]))
    gt = np.where(w.gt >= 0, o2n[np.maximum(w.gt, 0)], -1).astype(np.int32)
    return replace(w, graph=graph, entry=int(o2n[w.entry]), pq=pq, sq=sq, gt=gt, labels=None), new_to_old


def gorder_large(w, per_block: int = 32, threads: int | None = None):
    """The large workload's layout by gorder, clustered by the labels its
    build recorded (nearest mixture centre)."""
    n2o = gorder(w.graph, w.labels, int(w.labels.max()) + 1, per_block, threads=threads)
    return permute_large(w, n2o)
