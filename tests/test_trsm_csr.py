"""Z/p trsm with a sparse upper-triangular operand in CSR form: the GPU
counterpart of BLAS3::trsm on a SparseMatrix<uint32>, as Faugere-Lachartre
calls it for A^-1 B (lela/algorithms/faugere-lachartre.tcc:791).  The
solution of a triangular system with a unit diagonal is unique, so the
oracle's dense trsm on the same matrix is the expected result; singular
diagonals report the reference's index (the largest, for upper)."""
import numpy as np
import pytest

import oracle
from lela_b200 import gen, DiagonalEntryNotInvertible, PreconditionFailed


def _csr(D, extra_lower=0, seed=0):
    """CSR arrays of D (row-major, zeros dropped), plus `extra_lower` random
    entries left of the diagonal, which an upper solve must ignore."""
    g = np.random.default_rng(seed)
    n = D.shape[0]
    rows = []
    for r in range(n):
        cols = list(np.nonzero(D[r])[0])
        if extra_lower and r > 0:
            cols += list(g.choice(r, size=min(r, extra_lower), replace=False))
        cols = sorted(set(int(c) for c in cols))
        rows.append(cols)
    rowptr = np.zeros(n + 1, dtype=np.uint64)
    rowptr[1:] = np.cumsum([len(c) for c in rows])
    colidx = np.array([c for cs in rows for c in cs], dtype=np.uint32)
    vals = np.array([D[r, c] if c >= r else g.integers(1, 1000) for r, cs in enumerate(rows)
                     for c in cs], dtype=np.uint32)
    return rowptr, colidx, vals


def _sparse_upper(seed, n, p, unit, density=0.05):
    g = np.random.default_rng(seed)
    U = gen.upper_zp(seed, n, p, unit=unit)
    keep = g.random((n, n)) < density
    np.fill_diagonal(keep, True)
    return np.where(keep, U, 0).astype(np.uint32)


@pytest.mark.gpu
@pytest.mark.parametrize("p", [251, 65521, 2147483647, 4294967291])
def test_trsm_csr_upper_against_oracle(cuda, p):
    rng = np.random.default_rng(p % 991)
    for n, ncols in [(1, 1), (7, 3), (300, 50), (1100, 97)]:
        for unit in ((1,) if p >= 2**31 else (0, 1)):
            U = _sparse_upper(n + ncols, n, p, bool(unit))
            rowptr, colidx, vals = _csr(U, extra_lower=2, seed=n)
            B = gen.dense_zp(n * 3 + ncols, n, ncols, p)
            a = int(rng.integers(1, p))
            want, _ = oracle.trsm_zp(p, U, B, 1, unit, a)
            got = cuda.trsm_csr_upper(p, a, n, rowptr, colidx, vals, B.copy(), unit)
            assert np.array_equal(got, want), (p, n, ncols, unit)


@pytest.mark.gpu
def test_trsm_csr_upper_device_and_errors(cuda):
    import torch
    p, n, ncols = 65521, 600, 40
    U = _sparse_upper(3, n, p, False)
    rowptr, colidx, vals = _csr(U)
    B = gen.dense_zp(4, n, ncols, p)
    want, _ = oracle.trsm_zp(p, U, B, 1, 0, 1)
    dev = [torch.from_numpy(x.view(np.int64 if x.dtype == np.uint64 else np.int32)).cuda()
           for x in (rowptr, colidx, vals, B)]
    got = cuda.trsm_csr_upper(p, 1, n, dev[0], dev[1], dev[2], dev[3])
    cuda.synchronize()  # the device form runs on the handle's stream
    assert np.array_equal(got.cpu().numpy().view(np.uint32), want)
    # missing diagonal entries: the largest index is reported, B unchanged
    S = U.copy()
    S[100, 100] = 0
    S[450, 450] = 0
    rp, ci, va = _csr(S)
    X = B.copy()
    with pytest.raises(DiagonalEntryNotInvertible) as ei:
        cuda.trsm_csr_upper(p, 1, n, rp, ci, va, X)
    assert ei.value.idx == 450
    assert np.array_equal(X, B)
    # a column index past n
    bad = colidx.copy()
    bad[-1] = n
    with pytest.raises(PreconditionFailed):
        cuda.trsm_csr_upper(p, 1, n, rowptr, bad, vals, B.copy())
    bad_dev = torch.from_numpy(bad.view(np.int32)).cuda()
    with pytest.raises(PreconditionFailed):
        cuda.trsm_csr_upper(p, 1, n, dev[0], bad_dev, dev[2], dev[3].clone())


def _banded_upper(seed, n, p, unit, band, holes):
    """Upper triangular with nonzeros only within `band` columns right of the
    diagonal, minus square holes (row0, col0, size) -- the shape of F4 pivot
    blocks, whose 64 x 64 tiles away from the diagonal are mostly zero."""
    U = gen.upper_zp(seed, n, p, unit=unit)
    i, j = np.indices((n, n))
    U[(j - i) > band] = 0
    for r0, c0, s in holes:  # the diagonal stays (the system stays regular)
        hole = np.zeros((n, n), dtype=bool)
        hole[r0:r0 + s, c0:c0 + s] = True
        U[hole & (i != j)] = 0
    return U.astype(np.uint32)


@pytest.mark.gpu
@pytest.mark.parametrize("kernel", [1, 2])
@pytest.mark.parametrize("p", [65521, 2147483647])
def test_trsm_csr_upper_banded(cuda, kernel, p):
    """Banded sparse operands (most off-diagonal tiles empty): the updates
    are trimmed to the occupied tiles' bounding boxes; alpha != 1 (rows of
    B outside a box are only scaled), for both diagonal-block solvers."""
    from lela_b200 import api
    cuda.set_trsm_kernel(kernel)
    try:
        for n, ncols, band, holes in [(1500, 130, 300, [(0, 600, 400)]),
                                      (2600, 70, 700, [(1024, 1100, 300), (100, 400, 200)]),
                                      (700, 33, 0, [])]:
            U = _banded_upper(n + band, n, p, False, band, holes)
            rowptr, colidx, vals = _csr(U)
            B = gen.dense_zp(n + 7, n, ncols, p)
            for a in (1, 12345):
                want, _ = oracle.trsm_zp(p, U, B, 1, 0, a)
                got = cuda.trsm_csr_upper(p, a, n, rowptr, colidx, vals, B.copy(), False)
                assert np.array_equal(got, want), (kernel, p, n, band, a)
    finally:
        cuda.set_trsm_kernel(api.TRSM_AUTO)
