"""The benchmark workloads' k-means reduces without floating-point atomics
(datasets.cluster_sums), so every build of a workload gives the same
centroids, the same codebooks and the same graph."""
from __future__ import annotations

import numpy as np
import torch


def test_cluster_sums_match_a_float64_reduction():
    from rover_b200.datasets import cluster_sums
    g = torch.Generator().manual_seed(3)
    x = torch.randn(5000, 12, generator=g)
    labels = torch.randint(0, 40, (5000,), generator=g)
    labels[labels == 7] = 8                       # an empty cluster
    sums, cnt = cluster_sums(x, labels, 45)       # and clusters past the last label
    want = torch.zeros(45, 12, dtype=torch.float64).index_add_(0, labels, x.double())
    assert torch.allclose(sums.double(), want, rtol=1e-6, atol=1e-5)
    assert torch.equal(cnt, torch.bincount(labels, minlength=45).float())
    assert cnt[7] == 0 and torch.all(sums[7] == 0)


def test_training_is_repeatable():
    from rover_b200 import datasets as D
    base = D.gmm(3000, 16, 12, 5)
    a = D.train_pq(base, 4, 16, 5, device="cpu")
    b = D.train_pq(base, 4, 16, 5, device="cpu")
    assert np.array_equal(a, b)
    ca, la = D.kmeans_centroids(base, 12, iters=4, device="cpu")
    cb, lb = D.kmeans_centroids(base, 12, iters=4, device="cpu")
    assert np.array_equal(ca, cb) and np.array_equal(la, lb)


def test_representatives_are_each_clusters_nearest_member():
    from rover_b200.datasets import representatives
    g = torch.Generator().manual_seed(9)
    lab = torch.randint(0, 6, (400,), generator=g)
    lab[lab == 4] = 5                                # an empty cluster
    dc = torch.randint(0, 50, (400,), generator=g).float()   # with ties
    rep = representatives(dc, lab, 7)
    for j in range(7):
        members = torch.nonzero(lab == j).flatten()
        if len(members) == 0:
            assert rep[j] == -1
            continue
        best = members[dc[members] == dc[members].min()].min()   # nearest, then lowest id
        assert rep[j] == best
