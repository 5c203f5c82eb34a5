"""PQ codebook training and encoding on the GPU against the reference's own
C trainer and encoder (retrieval_pq_train / retrieval_pq_encode_batch,
retrieval_pq_core.c:97-268, compiled from the reference sources into
oracle/_ref and called directly): codebooks and codes bit for bit.

Shapes cover 8-bit codes (ks 256) and packed 4-bit codes (ks 16 with an odd
M), fewer training vectors than centroids (duplicate initial centroids, so
ties and empty clusters), a single training vector, zero iterations (run as
one, like the reference), the headline shape's M=16 x 256 over d=128, and the
refusal of non-finite training data.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

AEE_EBADPARM = 14


@pytest.fixture(scope="module")
def ref():
    from oracle import bindings
    if not bindings.reference_available():
        pytest.skip("oracle/_ref was not built (reference sources absent at build time)")
    return bindings.Reference()


def _mixture(n, dim, comps, seed):
    rng = np.random.default_rng(seed)
    centres = rng.normal(0, 2.0, size=(comps, dim))
    return (centres[rng.integers(0, comps, n)] + rng.normal(0, 0.5, size=(n, dim))).astype(np.float32)


@pytest.mark.parametrize("n,dim,m,ks,iters", [
    (3000, 32, 8, 256, 5),      # 8-bit codes
    (1500, 24, 6, 16, 10),      # 4-bit codes, even M
    (1200, 20, 5, 16, 6),       # 4-bit codes, odd M (half-filled last byte)
    (100, 16, 4, 256, 4),       # fewer vectors than centroids
    (1, 8, 2, 16, 3),           # one training vector
    (500, 16, 2, 64, 0),        # zero iterations run one
    (20000, 128, 16, 256, 8),   # the headline shape's codebook
])
def test_training_and_encoding_match_the_reference(calc, ref, n, dim, m, ks, iters):
    x = _mixture(n, dim, 12, n + dim)
    book = calc.pq_train(x, m, ks, iters)
    want = ref.pq_train(x, m, ks, iters)
    assert np.array_equal(book.view(np.uint32), want.view(np.uint32))
    probe = _mixture(4000, dim, 12, 7)
    assert np.array_equal(calc.pq_encode(probe, book), ref.pq_encode(probe, want))


def test_non_finite_training_data_is_refused(calc):
    from rover_b200.calculator import CalculatorError
    x = _mixture(100, 16, 4, 1)
    x[37, 5] = np.nan
    with pytest.raises(CalculatorError) as e:
        calc.pq_train(x, 4, 16, 2)
    assert e.value.code == AEE_EBADPARM
