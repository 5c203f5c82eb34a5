"""Seeded synthetic workloads with the shapes of the Rover configurations,
and the index-preparation steps that turn them into bundles.

The reference prepares bundles on a workstation (tools/index_bundle.py
prepare) from SIFT-like fvecs files; here a seeded Gaussian mixture stands in
for the dataset.  The preparation steps follow the reference writers:

* PQ codebook: per-subspace k-means from uniform-stride samples and
  uniform-stride initial centroids (tools/build_pure_pq_index.py:205-247);
  assignment ties go to the lowest centroid id.
* PQ codes: nearest centroid per subspace (build_pure_pq_index.py:326-351).
* PQ residual: per-vector min/max 4/8-bit quantization of
  raw - reconstruction, ``rint((r - min) / scale)``
  (tools/build_pure_pq_residual.py:137-158).
* SQ: global min/max L1 codes with round-half-away-from-zero, then per-vector
  residual codes (tools/encode_l1_residual.py:65-108).

Heavy steps (exact k-NN, pruning, k-means) run on the GPU through torch when
one is present; they are index preparation, not the search path.
"""
from __future__ import annotations

import numpy as np

try:
    import torch
except ImportError:  # pragma: no cover - torch is part of the image
    torch = None


def _device(device=None):
    if device is not None:
        return torch.device(device)
    return torch.device("cuda" if torch is not None and torch.cuda.is_available() else "cpu")


def gmm(n: int, dim: int, components: int, seed: int, sigma: float = 0.5, center_std: float = 2.0,
        clip_nonneg: bool = False, normalize: bool = False, centers_seed: int | None = None,
        return_centers: bool = False):
    """n points from a Gaussian mixture: centres ~ N(0, center_std^2 I) (drawn
    from ``centers_seed``, default ``seed``), per-component sigma, uniform
    component choice, float32."""
    crng = np.random.default_rng(seed if centers_seed is None else centers_seed)
    centers = crng.normal(0.0, center_std, size=(components, dim)).astype(np.float32)
    rng = np.random.default_rng([seed, 1])
    labels = rng.integers(0, components, size=n)
    x = rng.normal(0.0, sigma, size=(n, dim)).astype(np.float32)
    x += centers[labels]
    if clip_nonneg:
        np.maximum(x, 0.0, out=x)
    if normalize:
        x /= np.maximum(np.linalg.norm(x, axis=1, keepdims=True), np.float32(1e-12))
    x = np.ascontiguousarray(x, dtype=np.float32)
    return (x, centers) if return_centers else x


def exact_knn(queries: np.ndarray, base: np.ndarray, k: int, exclude_self: bool = False,
              device=None, chunk: int = 1024, margin: int = 16) -> np.ndarray:
    """Exact k nearest neighbours under squared L2, ties by lower id.
    Candidates come from an fp32 Gram-matrix pass (k + margin per row); the
    final order is recomputed from exact float64 differences."""
    dev = _device(device)
    with torch.no_grad():
        old_tf32 = torch.backends.cuda.matmul.allow_tf32
        torch.backends.cuda.matmul.allow_tf32 = False
        try:
            b = torch.from_numpy(np.ascontiguousarray(base)).to(dev)
            bn = (b * b).sum(1)
            kk = min(k + margin + (1 if exclude_self else 0), b.shape[0])
            chunk = max(16, min(chunk, (1 << 30) // max(1, b.shape[0])))   # distance block <= 4 GB
            out = np.empty((queries.shape[0], k), dtype=np.int32)
            for s in range(0, queries.shape[0], chunk):
                q = torch.from_numpy(np.ascontiguousarray(queries[s:s + chunk])).to(dev)
                d = bn[None, :] - 2.0 * (q @ b.T)
                if exclude_self:
                    rows = torch.arange(s, s + q.shape[0], device=dev)
                    d[torch.arange(q.shape[0], device=dev), rows] = float("inf")
                cand = torch.topk(d, kk, dim=1, largest=False).indices
                diff = q[:, None, :].double() - b[cand].double()
                exact = (diff * diff).sum(2)
                if exclude_self:
                    exact[cand == torch.arange(s, s + q.shape[0], device=dev)[:, None]] = float("inf")
                # lexicographic (distance, id): sort by id, then stable by distance
                idx_sorted, perm = torch.sort(cand, dim=1)
                exact = torch.gather(exact, 1, perm)
                order = torch.sort(exact, dim=1, stable=True).indices[:, :k]
                out[s:s + q.shape[0]] = torch.gather(idx_sorted, 1, order).cpu().numpy()
        finally:
            torch.backends.cuda.matmul.allow_tf32 = old_tf32
    return out


def alpha_prune(base: np.ndarray, candidates: np.ndarray, degree: int, alpha: float,
                device=None, chunk: int = 16384) -> np.ndarray:
    """Occlusion pruning of sorted candidate lists (DiskANN-style robust
    prune): walk candidates nearest first and keep c unless a kept k has
    alpha * d(k, c) <= d(p, c); keep at most ``degree``; pad with -1."""
    dev = _device(device)
    n, c = candidates.shape
    out = np.full((n, degree), -1, dtype=np.int32)
    with torch.no_grad():
        b = torch.from_numpy(np.ascontiguousarray(base)).to(dev)
        a2 = float(alpha) * float(alpha)
        for s in range(0, n, chunk):
            cand = torch.from_numpy(np.ascontiguousarray(candidates[s:s + chunk])).to(dev).long()
            p = b[s:s + cand.shape[0]]
            cv = b[cand.clamp_min(0)]
            dpc = ((cv - p[:, None, :]) ** 2).sum(2)
            dcc = torch.cdist(cv, cv) ** 2
            kept = torch.zeros_like(dpc, dtype=torch.bool)
            count = torch.zeros(cand.shape[0], dtype=torch.long, device=dev)
            valid = cand >= 0
            for i in range(c):
                occluded = (kept & (a2 * dcc[:, :, i] <= dpc[:, i:i + 1])).any(1)
                take = valid[:, i] & ~occluded & (count < degree)
                kept[:, i] = take
                count += take.long()
            rank = torch.cumsum(kept.long(), 1) - 1
            rows = torch.full((cand.shape[0], degree), -1, dtype=torch.long, device=dev)
            r_idx, c_idx = torch.nonzero(kept, as_tuple=True)
            rows[r_idx, rank[r_idx, c_idx]] = cand[r_idx, c_idx]
            out[s:s + cand.shape[0]] = rows.int().cpu().numpy()
    return out


def medoid(base: np.ndarray, device=None) -> int:
    """Index of the point nearest to the mean (the usual graph entry)."""
    dev = _device(device)
    with torch.no_grad():
        b = torch.from_numpy(np.ascontiguousarray(base)).to(dev)
        mean = b.double().mean(0)
        d = ((b.double() - mean) ** 2).sum(1)
        return int(torch.argmin(d).item())


def uniform_positions(population: int, count: int) -> np.ndarray:
    """tools/build_pure_pq_index.py:205-211."""
    if count == 1 or population == 1:
        return np.zeros(count, dtype=np.int64)
    return (np.arange(count, dtype=np.int64) * (population - 1)) // (count - 1)


def cluster_sums(x, labels, k: int):
    """Per-cluster sums and counts of x's rows, the same bits on every run:
    rows in label order (a stable sort), a float64 running sum, differences
    at the cluster boundaries -- no floating-point atomics, whose order (and
    so the k-means centroids, and the index built from them) would change
    from run to run."""
    order = torch.sort(labels, stable=True).indices
    cs = torch.cumsum(x[order].double(), 0)
    cnt = torch.bincount(labels, minlength=k)
    ends = torch.cumsum(cnt, 0)
    cs0 = torch.cat([torch.zeros((1, x.shape[1]), dtype=torch.float64, device=x.device), cs], 0)
    sums = cs0[ends] - cs0[ends - cnt]
    return sums.to(x.dtype), cnt.to(x.dtype)


def representatives(dc, lab, k: int):
    """rep[j] = the member of cluster j nearest its centre (dc: each point's
    distance to its own centre), ties to the lower id, -1 for an empty
    cluster.  Two stable sorts, no scatter with repeated indices (whose
    winning write the GPU does not fix)."""
    by_d = torch.sort(dc, stable=True).indices
    by_c = by_d[torch.sort(lab[by_d], stable=True).indices]
    cnt = torch.bincount(lab, minlength=k)
    start = torch.cumsum(cnt, 0) - cnt
    rep = torch.full((k,), -1, dtype=torch.long, device=dc.device)
    has = cnt > 0
    rep[has] = by_c[start[has]]
    return rep


def train_pq(base: np.ndarray, m: int, ks: int, iters: int, train_max: int = 100000,
             device=None) -> np.ndarray:
    """Per-subspace k-means codebook [m][ks][subdim] (float32)."""
    dev = _device(device)
    n, dim = base.shape
    subdim = dim // m
    sample = base[uniform_positions(n, min(n, train_max))]
    book = np.empty((m, ks, subdim), dtype=np.float32)
    with torch.no_grad():
        for s in range(m):
            x = torch.from_numpy(np.ascontiguousarray(sample[:, s * subdim:(s + 1) * subdim])).to(dev)
            cent = x[torch.from_numpy(uniform_positions(x.shape[0], ks)).to(dev)].clone()
            for _ in range(iters):
                d = ((x[:, None, :] - cent[None, :, :]) ** 2).sum(2) if x.shape[0] * ks <= (1 << 24) \
                    else torch.cdist(x, cent) ** 2
                a = torch.argmin(d, dim=1)
                sums, cnt = cluster_sums(x, a, ks)
                pop = cnt > 0
                cent[pop] = sums[pop] / cnt[pop, None]
            book[s] = cent.cpu().numpy()
    return book


def pq_encode(base: np.ndarray, book: np.ndarray, device=None, chunk: int = 1 << 16) -> np.ndarray:
    dev = _device(device)
    m, ks, subdim = book.shape
    n = base.shape[0]
    code_bytes = (m + 1) // 2 if ks == 16 else m
    codes = np.zeros((n, code_bytes), dtype=np.uint8)
    with torch.no_grad():
        cb = torch.from_numpy(book).to(dev)
        for s0 in range(0, n, chunk):
            x = torch.from_numpy(np.ascontiguousarray(base[s0:s0 + chunk])).to(dev)
            for s in range(m):
                xs = x[:, s * subdim:(s + 1) * subdim]
                d = ((xs[:, None, :] - cb[s][None, :, :]) ** 2).sum(2)
                a = torch.argmin(d, dim=1).to(torch.uint8).cpu().numpy()
                if ks == 16:
                    codes[s0:s0 + chunk, s // 2] |= (a << np.uint8(4)) if s & 1 else a
                else:
                    codes[s0:s0 + chunk, s] = a
    return codes


def pq_reconstruct(codes: np.ndarray, book: np.ndarray) -> np.ndarray:
    m, ks, subdim = book.shape
    out = np.empty((codes.shape[0], m * subdim), dtype=np.float32)
    for s in range(m):
        if ks == 16:
            a = (codes[:, s // 2] >> 4) if s & 1 else (codes[:, s // 2] & 0x0F)
        else:
            a = codes[:, s]
        out[:, s * subdim:(s + 1) * subdim] = book[s, a]
    return out


def quantize_residual_rint(residual: np.ndarray, bits: int):
    """tools/build_pure_pq_residual.py:137-158 (round half to even)."""
    levels = 15 if bits == 4 else 255
    mn = np.min(residual, axis=1).astype(np.float32)
    mx = np.max(residual, axis=1).astype(np.float32)
    scale = np.maximum((mx - mn) / np.float32(levels), np.float32(1.0e-12))
    q = np.rint((residual - mn[:, None]) / scale[:, None])
    q = np.clip(q, 0, levels).astype(np.uint8)
    return pack_codes(q, bits), np.column_stack((scale, mn)).astype(np.float32)


def pack_codes(q: np.ndarray, bits: int) -> np.ndarray:
    if bits == 8:
        return np.ascontiguousarray(q, dtype=np.uint8)
    n, d = q.shape
    packed = np.zeros((n, (d + 1) // 2), dtype=np.uint8)
    packed[:, :d // 2] = q[:, 0:d - 1:2] | (q[:, 1:d:2] << np.uint8(4))
    if d & 1:
        packed[:, -1] = q[:, -1]
    return packed


def _round_half_away(x: np.ndarray) -> np.ndarray:
    x = x.astype(np.float32)
    return (np.sign(x).astype(np.float32) * np.floor(np.abs(x) + np.float32(0.5)).astype(np.float32)).astype(np.float32)


def sq_encode(base: np.ndarray, l1_bits: int, residual_bits: int, chunk: int = 16384):
    """tools/encode_l1_residual.py:85-108, :140-200 restated: returns
    (l1_scale, l1_zero, l1_codes, residual_codes, qparams)."""
    eps = np.float32(1e-12)
    gmin = np.float32(base.min())
    gmax = np.float32(base.max())
    l1_scale = (np.maximum(gmax - gmin, eps) / np.float32((1 << l1_bits) - 1)).astype(np.float32)
    l1_zero = np.float32(gmin)
    inv = np.float32(1.0) / l1_scale
    l1_parts, res_parts, qp_parts = [], [], []
    for s in range(0, base.shape[0], chunk):
        x = base[s:s + chunk]
        q = np.clip(_round_half_away((x - l1_zero) * inv), 0, np.float32((1 << l1_bits) - 1)).astype(np.uint8)
        deq = (q.astype(np.float32) * l1_scale + l1_zero).astype(np.float32)
        r = (x - deq).astype(np.float32)
        rmin, rmax = r.min(axis=1), r.max(axis=1)
        rscale = (np.maximum(rmax - rmin, eps).astype(np.float32) / np.float32((1 << residual_bits) - 1)).astype(np.float32)
        rinv = (np.float32(1.0) / rscale).astype(np.float32)
        rq = np.clip(_round_half_away((r - rmin[:, None]) * rinv[:, None]), 0,
                     np.float32((1 << residual_bits) - 1)).astype(np.uint8)
        l1_parts.append(pack_codes(q, l1_bits))
        res_parts.append(pack_codes(rq, residual_bits))
        qp_parts.append(np.column_stack((rscale, rmin.astype(np.float32))).astype(np.float32))
    return (float(l1_scale), float(l1_zero), np.concatenate(l1_parts), np.concatenate(res_parts),
            np.concatenate(qp_parts))


def knn_graph(base: np.ndarray, degree: int, device=None) -> np.ndarray:
    """Exact degree-NN graph (no self edges; ties by lower id)."""
    return exact_knn(base, base, degree, exclude_self=True, device=device)


def pruned_graph(base: np.ndarray, candidates: int, degree: int, alpha: float, device=None) -> np.ndarray:
    """``candidates``-NN lists pruned by the alpha occlusion rule to at most
    ``degree`` neighbours (-1 padded)."""
    knn = exact_knn(base, base, candidates, exclude_self=True, device=device)
    return alpha_prune(base, knn, degree, alpha, device=device)


def pq_prepare(base: np.ndarray, m: int, ks: int, iters: int, residual_bits: int,
               train_max: int = 100000, device=None):
    """codebook, codes, residual rows and qparams for a pure-PQ bundle."""
    book = train_pq(base, m, ks, iters, train_max=train_max, device=device)
    codes = pq_encode(base, book, device=device)
    rows, qp = quantize_residual_rint(base - pq_reconstruct(codes, book), residual_bits)
    return book, codes, rows, qp


def kmeans_centroids(base: np.ndarray, k: int, iters: int = 10, device=None, seed: int = 0):
    """Plain Lloyd k-means (uniform-stride init); returns (centroids, labels)."""
    dev = _device(device)
    with torch.no_grad():
        x = torch.from_numpy(np.ascontiguousarray(base)).to(dev)
        # k-means++ seeding (D^2 sampling): separated clusters each get a centre
        gen = torch.Generator(device=dev)
        gen.manual_seed(seed)
        first = int(torch.randint(0, x.shape[0], (1,), generator=gen, device=dev).item())
        picks = [first]
        dmin = ((x - x[first]) ** 2).sum(1)
        for _ in range(1, k):
            r = torch.rand(1, generator=gen, device=dev) * dmin.sum()
            nxt = int(torch.searchsorted(torch.cumsum(dmin, 0), r).clamp_max(x.shape[0] - 1).item())
            picks.append(nxt)
            dmin = torch.minimum(dmin, ((x - x[nxt]) ** 2).sum(1))
        cent = x[torch.tensor(picks, device=dev)].clone()
        labels = None
        for _ in range(iters + 1):
            cn = (cent * cent).sum(1)
            parts = []
            for s in range(0, x.shape[0], 65536):
                xs = x[s:s + 65536]
                parts.append(torch.argmin(cn[None, :] - 2.0 * (xs @ cent.T), dim=1))
            labels = torch.cat(parts)
            sums, cnt = cluster_sums(x, labels, k)
            pop = cnt > 0
            cent[pop] = sums[pop] / cnt[pop, None]
        return cent.cpu().numpy(), labels.cpu().numpy()


def navigable_graph(base: np.ndarray, candidates: int, degree: int, alpha: float, long_edges: int = 8,
                    clusters: int | None = None, device=None, chunk: int = 16384) -> np.ndarray:
    """Occlusion-pruned k-NN graph plus long-range edges.

    A k-NN graph of well separated mixture data falls apart into one component
    per cluster, which no beam search can cross.  Here each node keeps at most
    ``degree - long_edges`` neighbours from its alpha-pruned k-NN list and
    spends the remaining slots on representatives (the member nearest the
    centroid) of the nearest other k-means clusters, each admitted only if no
    already kept neighbour occludes it (alpha * d(k, c) <= d(p, c))."""
    dev = _device(device)
    n = base.shape[0]
    clusters = clusters or max(16, int(np.sqrt(n)))
    intra = pruned_graph(base, candidates, degree - long_edges, alpha, device=device)
    cent, labels = kmeans_centroids(base, clusters, device=device)
    out = np.full((n, degree), -1, dtype=np.int32)
    out[:, :degree - long_edges] = intra
    with torch.no_grad():
        x = torch.from_numpy(np.ascontiguousarray(base)).to(dev)
        c = torch.from_numpy(cent).to(dev)
        lab = torch.from_numpy(labels).to(dev).long()
        # representative of each cluster: member nearest its centroid
        dc = ((x - c[lab]) ** 2).sum(1)
        rep = representatives(dc, lab, clusters)
        cn = (c * c).sum(1)
        a2 = float(alpha) * float(alpha)
        want = long_edges + 1
        for s in range(0, n, chunk):
            xs = x[s:s + chunk]
            b = xs.shape[0]
            near = torch.topk(cn[None, :] - 2.0 * (xs @ c.T), min(want, clusters), dim=1, largest=False).indices
            cand = rep[near]                                          # (b, want)
            ids = torch.arange(s, s + b, device=dev)
            cand = torch.where((cand == ids[:, None]) | (lab[s:s + b, None] == near), -1, cand)
            kept = torch.from_numpy(out[s:s + b]).to(dev).long()     # (b, degree)
            dpc = ((x[cand.clamp_min(0)] - xs[:, None, :]) ** 2).sum(2)  # (b, want)
            cnt = (kept >= 0).sum(1)
            for i in range(cand.shape[1]):
                ci = cand[:, i]
                cv = x[ci.clamp_min(0)]
                kv = x[kept.clamp_min(0)]
                dkc = ((kv - cv[:, None, :]) ** 2).sum(2)             # (b, degree)
                occl = ((kept >= 0) & (a2 * dkc <= dpc[:, i:i + 1])).any(1)
                dup = (kept == ci[:, None]).any(1)
                take = (ci >= 0) & ~occl & ~dup & (cnt < degree)
                rows = torch.nonzero(take, as_tuple=True)[0]
                kept[rows, cnt[rows]] = ci[rows]
                cnt = cnt + take.long()
            out[s:s + b] = kept.int().cpu().numpy()
    return out


def clustered_graph(base: np.ndarray, centers: np.ndarray, candidates: int, degree: int, alpha: float,
                    long_edges: int = 8, probe: int = 3, device=None, margin: int = 16) -> np.ndarray:
    """The navigable_graph recipe for indexes too large for an all-pairs
    k-NN pass: every point belongs to its nearest centre's cluster, and its
    ``candidates`` nearest neighbours are searched among the members of its
    own cluster and of the ``probe - 1`` clusters whose centres are nearest
    that cluster's centre (a TF32 Gram pass picks candidates + margin, exact
    float32 differences order them, ties by lower id).  The lists are
    alpha-pruned to ``degree - long_edges`` neighbours, and the remaining
    slots hold representatives (the member nearest the centre) of the
    nearest other clusters, each admitted only if no kept neighbour occludes
    it (alpha * d(k, c) <= d(p, c)).  Fixture construction, not the search
    path."""
    dev = _device(device)
    n, dim = base.shape
    k_clusters = centers.shape[0]
    knn = np.full((n, candidates), -1, dtype=np.int32)
    with torch.no_grad():
        x = torch.from_numpy(np.ascontiguousarray(base)).to(dev)
        c = torch.from_numpy(np.ascontiguousarray(centers, dtype=np.float32)).to(dev)
        cn = (c * c).sum(1)
        labels = torch.empty(n, dtype=torch.long, device=dev)
        for s in range(0, n, 1 << 16):
            labels[s:s + (1 << 16)] = torch.argmin(cn[None, :] - 2.0 * (x[s:s + (1 << 16)] @ c.T), dim=1)
        order = torch.argsort(labels, stable=True)
        counts = torch.bincount(labels, minlength=k_clusters)
        starts = torch.cumsum(counts, 0) - counts
        near = torch.topk(torch.cdist(c, c), min(probe, k_clusters), dim=1, largest=False).indices
        counts_h, starts_h, near_h = counts.cpu().numpy(), starts.cpu().numpy(), near.cpu().numpy()
        old_tf32 = torch.backends.cuda.matmul.allow_tf32
        torch.backends.cuda.matmul.allow_tf32 = True
        try:
            for cl in range(k_clusters):
                if counts_h[cl] == 0:
                    continue
                mine = order[starts_h[cl]:starts_h[cl] + counts_h[cl]]
                pool = torch.cat([order[starts_h[o]:starts_h[o] + counts_h[o]] for o in near_h[cl]])
                q, b = x[mine], x[pool]
                d = (b * b).sum(1)[None, :] - 2.0 * (q @ b.T)
                d[mine[:, None] == pool[None, :]] = float("inf")
                kk = min(candidates + margin, pool.shape[0])
                cand = pool[torch.topk(d, kk, dim=1, largest=False).indices]
                diff = q[:, None, :] - x[cand]
                exact = (diff * diff).sum(2)
                exact[cand == mine[:, None]] = float("inf")
                ids_sorted, perm = torch.sort(cand, dim=1)
                exact = torch.gather(exact, 1, perm)
                pick = torch.sort(exact, dim=1, stable=True).indices[:, :candidates]
                best = torch.gather(ids_sorted, 1, pick)
                bad = torch.gather(exact, 1, pick) == float("inf")
                best[bad] = -1
                got = best.shape[1]
                knn[mine.cpu().numpy(), :got] = best.int().cpu().numpy()
        finally:
            torch.backends.cuda.matmul.allow_tf32 = old_tf32
    intra = alpha_prune(base, knn, degree - long_edges, alpha, device=device)
    out = np.full((n, degree), -1, dtype=np.int32)
    out[:, :degree - long_edges] = intra
    with torch.no_grad():
        lab = labels
        dc = ((x - c[lab]) ** 2).sum(1)
        rep = representatives(dc, lab, k_clusters)
        a2 = float(alpha) * float(alpha)
        want = long_edges + 1
        chunk = 16384
        for s in range(0, n, chunk):
            xs = x[s:s + chunk]
            bsz = xs.shape[0]
            nc = torch.topk(cn[None, :] - 2.0 * (xs @ c.T), min(want, k_clusters), dim=1, largest=False).indices
            cand = rep[nc]
            ids = torch.arange(s, s + bsz, device=dev)
            cand = torch.where((cand == ids[:, None]) | (lab[s:s + bsz, None] == nc) | (cand < 0), -1, cand)
            kept = torch.from_numpy(out[s:s + bsz]).to(dev).long()
            dpc = ((x[cand.clamp_min(0)] - xs[:, None, :]) ** 2).sum(2)
            cnt = (kept >= 0).sum(1)
            for i in range(cand.shape[1]):
                ci = cand[:, i]
                cv = x[ci.clamp_min(0)]
                kv = x[kept.clamp_min(0)]
                dkc = ((kv - cv[:, None, :]) ** 2).sum(2)
                occl = ((kept >= 0) & (a2 * dkc <= dpc[:, i:i + 1])).any(1)
                dup = (kept == ci[:, None]).any(1)
                take = (ci >= 0) & ~occl & ~dup & (cnt < degree)
                rows = torch.nonzero(take, as_tuple=True)[0]
                kept[rows, cnt[rows]] = ci[rows]
                cnt = cnt + take.long()
            out[s:s + bsz] = kept.int().cpu().numpy()
        del x
    return out


def routed_graph(base: np.ndarray, candidates: int, degree: int, alpha: float, long_edges: int = 8,
                 clusters: int | None = None, entry: int | None = None, device=None) -> tuple[np.ndarray, int]:
    """``navigable_graph`` plus a two-level routing structure so that a beam
    search from the entry can reach every cluster.  Routing rows hold only
    cluster representatives (the member nearest each k-means centroid): the
    entry's row lists ``degree`` hub nodes, each hub's row lists its share of
    all representatives.  Hubs are ordinary nodes that are not
    representatives; their clusters stay connected through the other members.
    Returns (graph, entry)."""
    dev = _device(device)
    n = base.shape[0]
    clusters = clusters or max(16, int(np.sqrt(n)))
    graph = navigable_graph(base, candidates, degree, alpha, long_edges, clusters, device)
    cent, labels = kmeans_centroids(base, clusters, device=device)
    entry = medoid(base, device) if entry is None else entry
    with torch.no_grad():
        x = torch.from_numpy(np.ascontiguousarray(base)).to(dev)
        c = torch.from_numpy(cent).to(dev)
        lab = torch.from_numpy(labels).to(dev).long()
        dc = ((x - c[lab]) ** 2).sum(1)
        rep = representatives(dc, lab, clusters)
        reps = [int(r) for r in rep.cpu().numpy() if r >= 0 and r != entry]
        # hubs: the nodes nearest the entry that are not representatives
        taken = set(reps) | {entry}
        near = torch.argsort(((x - x[entry]) ** 2).sum(1))[: degree + len(taken) + 1].cpu().numpy()
        hubs = [int(v) for v in near if int(v) not in taken][:degree]
    per = (len(reps) + len(hubs) - 1) // max(1, len(hubs))
    if per > degree:
        raise ValueError("too many clusters for a two-level routing of this degree")
    graph[entry, :] = -1
    graph[entry, :len(hubs)] = hubs
    for h_i, h in enumerate(hubs):
        mine = reps[h_i * per:(h_i + 1) * per]
        graph[h, :] = -1
        graph[h, :len(mine)] = mine
    return graph, entry
