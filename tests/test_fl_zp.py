"""Faugere-Lachartre on the GPU against LELA's results -- the counterpart of
tests/test-faugere-lachartre.C:179-247 (FL output equals the reduced echelon
form, ranks agree), run over Modular<uint32> (which the reference test does
not exercise) in all four modes, bit-exact in R, rank and det."""
import types

import numpy as np
import pytest

import golden_io
import oracle
from lela_b200 import gen, WrongMatrixForm

MODES = ((1, 0), (0, 0), (1, 1), (0, 1))


@pytest.mark.gpu
def test_fl_golden(cuda):
    for (pre, p, m, n, red, od, st, rank, det, rowptr, colidx, vals, R) in golden_io.fl_cases():
        X = gen.CSR(m, n, rowptr, colidx, vals)
        got, gr, gd = cuda.fl_echelonize(p, X, red, od)
        assert (gr, gd) == (rank, det), pre
        assert np.array_equal(got, R), pre


@pytest.mark.gpu
def test_fl_golden_f4_digest(cuda):
    z, man = golden_io.data()
    X = gen.f4_matrix(7, 300, 65521, density=0.03)
    for pre in man["fl"]:
        if pre + "R_sha" not in man:
            continue
        _, _, _, red, od, st, rank, det = (int(x) for x in z[pre + "meta"])
        got, gr, gd = cuda.fl_echelonize(65521, X, red, od)
        assert (gr, gd) == (rank, det), pre
        assert golden_io.sha(np.ascontiguousarray(got)) == man[pre + "R_sha"], pre


@pytest.mark.gpu
@pytest.mark.parametrize("seed", range(3))
def test_fl_f4_shaped_against_oracle(cuda, seed):
    p = 65521
    for m in (200, 700, 1500):
        X = gen.f4_matrix(100 * seed + m, m, p)
        for red, od in MODES:
            want = oracle.fl_echelonize_zp(p, X.m, X.n, X.rowptr, X.colidx, X.vals, red, od)
            got, gr, gd = cuda.fl_echelonize(p, X, red, od)
            assert (gr, gd) == (want["rank"], want["det"]), (m, red, od)
            assert np.array_equal(got, want["R"]), (m, red, od)


@pytest.mark.gpu
@pytest.mark.parametrize("p", [251, 65521, 2147483647])
def test_fl_reference_family(cuda, p):
    """The reference test's staircase family (tests/test-faugere-lachartre.C:
    142-175) at several sizes and densities."""
    for seed, (m, n, dens) in enumerate([(96, 128, 0.1), (300, 280, 0.05), (500, 900, 0.02)]):
        X = gen.f4_matrix_small(seed, m, n, p, dens)
        for red, od in MODES:
            want = oracle.fl_echelonize_zp(p, X.m, X.n, X.rowptr, X.colidx, X.vals, red, od)
            got, gr, gd = cuda.fl_echelonize(p, X, red, od)
            assert (gr, gd) == (want["rank"], want["det"]), (p, m, n, red, od)
            assert np.array_equal(got, want["R"]), (p, m, n, red, od)


@pytest.mark.gpu
def test_fl_edge_cases(cuda):
    p = 65521
    # WrongMatrixForm at the row whose head lies left of the previous pivot
    D = np.zeros((4, 6), dtype=np.uint32)
    D[0, 1] = 1; D[1, 3] = 1; D[2, 2] = 5; D[3, 4] = 1
    with pytest.raises(WrongMatrixForm) as ei:
        cuda.fl_echelonize(p, gen.CSR.from_dense(D))
    assert ei.value.row == 2
    # all rows empty; a single row; no non-pivot rows; only non-pivot rows after an empty row
    T = np.triu(gen.dense_zp(1, 6, 8, p), 0)
    T[np.arange(6), np.arange(6)] = np.maximum(T[np.arange(6), np.arange(6)], 1)
    for D in (np.zeros((3, 5), np.uint32), np.array([[0, 4, 0, 7]], np.uint32), T,
              np.array([[1, 2, 0], [0, 0, 0], [0, 3, 1], [1, 1, 1]], np.uint32)):
        X = gen.CSR.from_dense(D)
        for red, od in MODES:
            want = oracle.fl_echelonize_zp(p, X.m, X.n, X.rowptr, X.colidx, X.vals, red, od)
            got, gr, gd = cuda.fl_echelonize(p, X, red, od)
            assert want["status"] == 0
            assert (gr, gd) == (want["rank"], want["det"]), (D.shape, red, od)
            assert np.array_equal(got, want["R"]), (D.shape, red, od)


@pytest.mark.gpu
def test_fl_device_path(cuda):
    import torch
    p = 65521
    X = gen.f4_matrix(5, 600, p)
    want = oracle.fl_echelonize_zp(p, X.m, X.n, X.rowptr, X.colidx, X.vals, 1, 0)
    T = types.SimpleNamespace(m=X.m, n=X.n,
                              rowptr=torch.from_numpy(X.rowptr.view(np.int64)).cuda(),
                              colidx=torch.from_numpy(X.colidx.view(np.int32)).cuda(),
                              vals=torch.from_numpy(X.vals.view(np.int32)).cuda())
    R, gr, gd = cuda.fl_echelonize(p, T, True, False)
    torch.cuda.synchronize()
    assert (gr, gd) == (want["rank"], want["det"])
    assert np.array_equal(R.cpu().numpy().view(np.uint32), want["R"])


@pytest.mark.gpu
@pytest.mark.parametrize("red,od", MODES)
def test_fl_csr_output(cuda, red, od):
    """The CSR form of the result (the SparseMatrix the reference writes)
    against the dense one and the oracle: same rows, column indices strictly
    increasing, every stored value nonzero; host and device paths; a first
    guess of the capacity that is too small (the kept result is fetched)."""
    import torch
    p = 65521
    for seed, m in ((1, 900), (2, 1500)):
        X = gen.f4_matrix(300 + seed, m, p)
        want = oracle.fl_echelonize_zp(p, X.m, X.n, X.rowptr, X.colidx, X.vals, red, od)
        for cap in (None, 5):
            R, gr, gd = cuda.fl_echelonize_csr(p, X, red, od, cap=cap)
            assert (gr, gd) == (want["rank"], want["det"]), (m, red, od, cap)
            assert R.m == want["R"].shape[0]
            assert np.array_equal(R.to_dense(), want["R"]), (m, red, od, cap)
            rows = np.repeat(np.arange(R.m), np.diff(R.rowptr).astype(np.int64))
            d = np.diff(R.colidx.astype(np.int64))
            assert (d[rows[1:] == rows[:-1]] > 0).all()
            assert (R.vals != 0).all()
        T = types.SimpleNamespace(m=X.m, n=X.n,
                                  rowptr=torch.from_numpy(X.rowptr.view(np.int64)).cuda(),
                                  colidx=torch.from_numpy(X.colidx.view(np.int32)).cuda(),
                                  vals=torch.from_numpy(X.vals.view(np.int32)).cuda())
        Rd, gr, gd = cuda.fl_echelonize_csr(p, T, red, od, cap=7)
        torch.cuda.synchronize()
        assert (gr, gd) == (want["rank"], want["det"])
        Rh = gen.CSR(Rd.m, X.n, Rd.rowptr.cpu().numpy().view(np.uint64),
                     Rd.colidx.cpu().numpy().view(np.uint32), Rd.vals.cpu().numpy().view(np.uint32))
        assert np.array_equal(Rh.to_dense(), want["R"])


@pytest.mark.gpu
def test_fl_csr_edge_cases(cuda):
    """Empty results (all rows zero; no D rows with only_D) and the fetch
    without a kept result."""
    p = 65521
    for D in (np.zeros((3, 5), np.uint32), np.array([[0, 4, 0, 7]], np.uint32)):
        X = gen.CSR.from_dense(D)
        for red, od in MODES:
            want = oracle.fl_echelonize_zp(p, X.m, X.n, X.rowptr, X.colidx, X.vals, red, od)
            R, gr, gd = cuda.fl_echelonize_csr(p, X, red, od)
            assert (gr, gd) == (want["rank"], want["det"])
            assert np.array_equal(R.to_dense(), want["R"].reshape(R.m, X.n)), (D.shape, red, od)
