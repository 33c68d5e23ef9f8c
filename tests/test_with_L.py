"""The echelon forms with L that are composed from the GPU's standard
transform (tests/test_echelon_transform.py): GaussJordan::echelonize_reduced
with its transform (lela/algorithms/gauss-jordan.tcc:434-466), and the
non-reduced forms that keep L below the diagonal, Elimination::echelonize
with its default compute_L (lela/algorithms/elimination.tcc:47-139) and
GaussJordan::echelonize (gauss-jordan.tcc:413-432), against LELA's own
results (tests/golden/make_transform_golden.py) and the oracle's
restatements, bit-exact in the matrix, P, rank and det."""
import numpy as np
import pytest

import golden_io
import oracle
from lela_b200 import gen, LELAError
from lela_b200.api import PreconditionFailed


def _kind(A, p, kind, seed):
    m, n = A.shape
    if kind == 1:
        A[:, ::3] = 0
    elif kind == 2:
        r = max(1, min(m, n) // 3)
        F = (gen.dense_zp(seed, m, r, p).astype(object) @ gen.dense_zp(seed + 1, r, n, p).astype(object)) % p
        A = F.astype(np.uint32)
    elif kind == 3:
        A[m // 2:] = 0
        A[:, :n // 2] = 0
    return A


@pytest.mark.gpu
def test_gj_transform_golden(cuda):
    """GaussJordan::echelonize_reduced with its transform (pivots keep their
    values) against LELA's own results."""
    n = 0
    for pre, p, st, r, d, A, R, L, P in golden_io.transform_cases(gj=True):
        if p >= 2 ** 31:
            with pytest.raises(PreconditionFailed):
                cuda.echelon_reduced_transform(p, A.copy(), unit_pivots=False)
            continue
        if st:
            with pytest.raises(LELAError):
                cuda.echelon_reduced_transform(p, A.copy(), unit_pivots=False)
            continue
        gR, gL, gP, gr, gd = cuda.echelon_reduced_transform(p, A.copy(), unit_pivots=False)
        assert (gr, gd) == (r, d) and gP == P, pre
        assert np.array_equal(gR, R) and np.array_equal(gL, L), pre
        n += 1
    assert n >= 70


@pytest.mark.gpu
@pytest.mark.parametrize("p", [3, 65521, 2147483647])
def test_gj_transform_against_oracle(cuda, p):
    rng = np.random.default_rng(p % 907)
    for (m, n) in ((1, 1), (7, 13), (13, 7), (130, 70), (300, 300)):
        for kind in range(4):
            seed = int(rng.integers(1 << 30))
            A = _kind(gen.dense_zp(seed, m, n, p), p, kind, seed + 1)
            want = oracle.gj_echelon_reduced_L_zp(p, A)
            R, L, P, r, d = cuda.echelon_reduced_transform(p, A.copy(), unit_pivots=False)
            tag = (p, m, n, kind)
            assert (r, d) == (want[3], want[4]) and P == want[2], tag
            assert np.array_equal(R, want[0]) and np.array_equal(L, want[1]), tag


@pytest.mark.gpu
def test_packed_L_golden(cuda):
    """Elimination::echelonize with its default compute_L and GaussJordan::
    echelonize (L kept below the diagonal) against LELA's own results."""
    n = 0
    for pre, gj, p, st, r, d, A, E, P in golden_io.packed_cases():
        if p >= 2 ** 31:
            with pytest.raises(PreconditionFailed):
                cuda.echelonize_with_L(p, A.copy(), gauss_jordan=gj)
            continue
        if st:
            with pytest.raises(LELAError):
                cuda.echelonize_with_L(p, A.copy(), gauss_jordan=gj)
            continue
        gE, gP, gr, gd = cuda.echelonize_with_L(p, A.copy(), gauss_jordan=gj)
        assert (gr, gd) == (r, d) and gP == P, (pre, gj)
        assert np.array_equal(gE, E), (pre, gj)
        n += 1
    assert n >= 140


@pytest.mark.gpu
@pytest.mark.parametrize("p", [3, 65521, 2147483647])
def test_packed_L_against_oracle(cuda, p):
    rng = np.random.default_rng(p % 887)
    for (m, n) in ((1, 1), (7, 13), (13, 7), (130, 70), (70, 130), (300, 300)):
        for kind in range(4):
            seed = int(rng.integers(1 << 30))
            A = _kind(gen.dense_zp(seed, m, n, p), p, kind, seed + 1)
            for gj in (False, True):
                want = oracle.echelon_packed_L_zp(p, A, gj)
                E, P, r, d = cuda.echelonize_with_L(p, A.copy(), gauss_jordan=gj)
                tag = (p, m, n, kind, gj)
                assert (r, d) == (want[2], want[3]) and P == want[1], tag
                assert np.array_equal(E, want[0]), tag
