"""Dense Z/p row-echelon form on the GPU against LELA's results: the
counterpart of tests/test-gauss-jordan.C:91-99 (GaussJordan + move_L equals
Elimination::echelonize) and tests/test-elimination.C.  The non-reduced form
and det depend on the pivot rule, so these compare U, rank and det exactly,
including inputs that force the non-generic paths (zero columns, zero and
dependent rows, tiny moduli with many zero pivots)."""
import numpy as np
import pytest

import golden_io
import oracle
from lela_b200 import gen, LELAError


@pytest.mark.gpu
def test_echelon_golden(cuda):
    for pre, p, st, r, d, A, E in golden_io.echelon_cases():
        if st:
            with pytest.raises(LELAError):
                cuda.echelonize(p, A.copy())
            continue
        got, gr, gd = cuda.echelonize(p, A.copy())
        assert (gr, gd) == (r, d), pre
        assert np.array_equal(got, E), pre


def _structured(seed, m, n, p):
    g = np.random.default_rng(seed)
    A = gen.dense_zp(seed, m, n, p)
    A[:, g.choice(n, size=max(1, n // 10), replace=False)] = 0        # zero columns
    A[g.choice(m, size=max(1, m // 10), replace=False)] = 0           # zero rows
    deps = g.choice(m, size=max(1, m // 8), replace=False) if m >= 2 else []
    for r in deps:                                                    # dependent rows
        a, b = g.choice(m, size=2, replace=False)
        A[r] = (A[a].astype(np.uint64) * 3 + A[b].astype(np.uint64) * 5) % p
    k = min(3, n)
    A[:, :k] = np.where(g.random((m, k)) < 0.7, 0, A[:, :k])          # sparse leading columns
    return A


@pytest.mark.gpu
@pytest.mark.parametrize("p", [2, 3, 251, 65521, 2147483647])
def test_echelon_against_oracle(cuda, p):
    for seed, (m, n) in enumerate([(1, 1), (5, 9), (64, 64), (65, 130), (200, 90), (150, 400), (333, 333)]):
        for kind in ("dense", "structured"):
            A = gen.dense_zp(seed, m, n, p) if kind == "dense" else _structured(seed, m, n, p)
            want, wr, wd = oracle.echelon_zp(p, A)
            got, gr, gd = cuda.echelonize(p, A.copy())
            assert (gr, gd) == (wr, wd), (p, m, n, kind)
            assert np.array_equal(got, want), (p, m, n, kind)


@pytest.mark.gpu
def test_echelon_large(cuda):
    """A 1500 x 2200 rank-deficient matrix (p = 65521)."""
    p = 65521
    A = _structured(77, 1500, 2200, p)
    want, wr, wd = oracle.echelon_zp(p, A)
    got, gr, gd = cuda.echelonize(p, A.copy())
    assert (gr, gd) == (wr, wd)
    assert np.array_equal(got, want)


@pytest.mark.gpu
@pytest.mark.parametrize("p", [3, 65521])
def test_echelon_pivots_far_below(cuda, p):
    """Pivots that lie hundreds of rows below the current row: the first 700
    rows are zero in the leading columns, so the search reaches rows beyond
    the block it keeps on chip, and the transpositions move rows across it."""
    g = np.random.default_rng(5)
    m, n = 1200, 150
    A = gen.dense_zp(91, m, n, p)
    A[:700, :40] = 0
    A[g.choice(np.arange(700, m), size=300, replace=False), :12] = 0
    A[::7, 70:75] = 0
    want, wr, wd = oracle.echelon_zp(p, A)
    got, gr, gd = cuda.echelonize(p, A.copy())
    assert (gr, gd) == (wr, wd)
    assert np.array_equal(got, want)


@pytest.mark.gpu
@pytest.mark.parametrize("p", [3, 2147483647])
def test_echelon_blocks_far_pivots(cuda, p):
    """Several blocks of panels (delayed trailing updates) with pivots far
    below the current row across block boundaries, a block-wide band of zero
    columns, dependent rows and rows that become zero mid-block."""
    g = np.random.default_rng(11)
    m, n = 1100, 900
    A = gen.dense_zp(17, m, n, p)
    A[:600, :300] = 0                      # the first block's pivots lie far below
    A[:, 400:470] = 0                      # a panel and more without pivots
    A[g.choice(np.arange(600, m), size=200, replace=False), :20] = 0
    for r in g.choice(m, size=60, replace=False):
        a, b = g.choice(m, size=2, replace=False)
        A[r] = (A[a].astype(np.uint64) * 2 + A[b].astype(np.uint64) * 7) % p
    want, wr, wd = oracle.echelon_zp(p, A)
    got, gr, gd = cuda.echelonize(p, A.copy())
    assert (gr, gd) == (wr, wd)
    assert np.array_equal(got, want)


# ------------------------------------------------------------ reduced form
# EchelonForm::echelonize (A, true) on a DenseMatrix: GaussJordan::
# echelonize_reduced (lela/algorithms/gauss-jordan.tcc:434-466).

@pytest.mark.gpu
@pytest.mark.parametrize("unit", [False, True])
def test_echelon_reduced_golden(cuda, unit):
    """unit: the standard method's form (Elimination::echelonize_reduced,
    lela/algorithms/elimination.tcc:143-265), pivots scaled to 1."""
    for pre, p, st, r, d, A, E in golden_io.echelon_reduced_cases(unit):
        if st:
            with pytest.raises(LELAError):
                cuda.echelonize(p, A.copy(), reduced=True, unit_pivots=unit)
            continue
        got, gr, gd = cuda.echelonize(p, A.copy(), reduced=True, unit_pivots=unit)
        assert (gr, gd) == (r, d), pre
        assert np.array_equal(got, E), pre


@pytest.mark.gpu
@pytest.mark.parametrize("p", [2, 3, 251, 65521, 2147483647])
def test_echelon_reduced_against_oracle(cuda, p):
    for seed, (m, n) in enumerate([(1, 1), (5, 9), (9, 5), (64, 64), (65, 130), (200, 90),
                                   (150, 400), (333, 333)]):
        for kind in ("dense", "structured"):
            A = gen.dense_zp(seed, m, n, p) if kind == "dense" else _structured(seed, m, n, p)
            for unit in (False, True):
                want, wr, wd = oracle.echelon_reduced_zp(p, A, unit)
                got, gr, gd = cuda.echelonize(p, A.copy(), reduced=True, unit_pivots=unit)
                assert (gr, gd) == (wr, wd), (p, m, n, kind, unit)
                assert np.array_equal(got, want), (p, m, n, kind, unit)


@pytest.mark.gpu
def test_echelon_reduced_large(cuda):
    """1400 x 1600, rank about 1090: the pivot block is solved through the
    inverted 512-row diagonal blocks on the tensor cores."""
    p = 65521
    A = _structured(78, 1400, 1600, p)
    want, wr, wd = oracle.echelon_reduced_zp(p, A)
    assert wr >= 1024
    got, gr, gd = cuda.echelonize(p, A.copy(), reduced=True)
    assert (gr, gd) == (wr, wd)
    assert np.array_equal(got, want)


@pytest.mark.gpu
def test_echelon_reduced_device(cuda):
    """The _dev entry point on a torch CUDA view with a row stride."""
    import torch
    p = 251
    A = _structured(79, 120, 170, p)
    want, wr, wd = oracle.echelon_reduced_zp(p, A)
    big = torch.zeros((120, 200), dtype=torch.int32, device="cuda")
    big[:, 10:180] = torch.from_numpy(A.view(np.int32)).cuda()
    view = big[:, 10:180]
    _, gr, gd = cuda.echelonize(p, view, reduced=True)
    cuda.synchronize()
    host = big.cpu().numpy().view(np.uint32)
    assert (gr, gd) == (wr, wd)
    assert np.array_equal(host[:, 10:180], want)
    assert not host[:, :10].any() and not host[:, 180:].any()
