"""The standard method's reduced form with its transform on the GPU against
LELA's Elimination::echelonize_reduced (A, L, P, rank, det, compute_L =
true) (lela/algorithms/elimination.tcc:143-265): the golden fixtures LELA
computed and the oracle's step-by-step restatement, bit-exact in R, L, the
transposition list, rank and det.  At sizes with several delayed panel
blocks the result is checked by its defining properties: R equals the GPU's
reduced form (itself checked against the oracle), P equals the PLUQ row
transpositions, L has the block form [[X, 0], [Y, I]], and R = L P A by
random projections (which with that block form determines L)."""
import numpy as np
import pytest

import golden_io
import oracle
from lela_b200 import gen, LELAError
from lela_b200.api import PreconditionFailed


def _check(cuda, p, A, tag):
    try:
        want = oracle.echelon_reduced_L_zp(p, A)
    except ArithmeticError:
        want = None
    if want is None:
        with pytest.raises(LELAError):
            cuda.echelon_reduced_transform(p, A.copy())
        return
    R, L, P, r, d = cuda.echelon_reduced_transform(p, A.copy())
    assert (r, d) == (want[3], want[4]), tag
    assert P == want[2], tag
    assert np.array_equal(R, want[0]), tag
    assert np.array_equal(L, want[1]), tag


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
def test_transform_golden(cuda):
    n = 0
    for pre, p, st, r, d, A, R, L, P in golden_io.transform_cases():
        if p >= 2 ** 31:
            # Modular<uint32>'s inverse wraps above 2^31: no transform exists
            with pytest.raises(PreconditionFailed):
                cuda.echelon_reduced_transform(p, A.copy())
            continue
        if st:
            with pytest.raises(LELAError):
                cuda.echelon_reduced_transform(p, A.copy())
            continue
        gR, gL, gP, gr, gd = cuda.echelon_reduced_transform(p, A.copy())
        assert (gr, gd) == (r, d) and gP == P, pre
        assert np.array_equal(gR, R) and np.array_equal(gL, L), pre
        n += 1
    assert n >= 70


@pytest.mark.gpu
@pytest.mark.parametrize("p", [2, 3, 251, 65521, 65536, 2147483647])
def test_transform_against_oracle(cuda, p):
    rng = np.random.default_rng(p % 919)
    for (m, n) in ((1, 1), (2, 9), (7, 13), (13, 7), (70, 130), (130, 70), (300, 300), (520, 470)):
        for kind in range(4):
            seed = int(rng.integers(1 << 30))
            A = _kind(gen.dense_zp(seed, m, n, p), p, kind, seed + 1)
            _check(cuda, p, A, (p, m, n, kind))


@pytest.mark.gpu
def test_transform_empty(cuda):
    p = 65521
    for (m, n) in ((0, 0), (0, 6), (6, 0)):
        R, L, P, r, d = cuda.echelon_reduced_transform(p, np.zeros((m, n), dtype=np.uint32))
        assert (r, d, P) == (0, 1, []) and R.shape == (m, n)
        assert np.array_equal(L, np.eye(m, dtype=np.uint32))


def _project_check(p, A, R, L, P, r, seed):
    """L has the block form [[X, 0], [Y, I]] and R = L P A (two random
    projections, exact integer arithmetic)."""
    m = A.shape[0]
    assert not L[:r, r:].any()
    assert np.array_equal(L[r:, r:], np.eye(m - r, dtype=np.uint32))
    B = A.copy()
    for a, b in P:
        B[[a, b]] = B[[b, a]]
    rng = np.random.default_rng(seed)
    for _ in range(2):
        x = rng.integers(0, p, A.shape[1]).astype(object)
        lhs = R.astype(object).dot(x) % p
        rhs = L.astype(object).dot(B.astype(object).dot(x) % p) % p
        assert np.array_equal(lhs, rhs)


@pytest.mark.gpu
@pytest.mark.parametrize("p", [65521, 2147483647])
def test_transform_blocks_and_far_pivots(cuda, p):
    """Several 64-column panels in delayed blocks (more than 512 rows below
    the first pivots), pivots far below the current row, a zero column band
    and a rank-deficient tall matrix."""
    cases = []
    A = gen.dense_zp(31, 1600, 1200, p)
    cases.append(("dense 1600x1200", A))
    B = gen.dense_zp(32, 1500, 900, p)
    B[:1100, :70] = 0
    cases.append(("far pivots", B))
    C = gen.dense_zp(33, 900, 1400, p)
    C[:, 200:330] = 0
    cases.append(("zero column band", C))
    F = (gen.dense_zp(34, 1300, 400, p).astype(object) @ gen.dense_zp(35, 400, 1000, p).astype(object)) % p
    cases.append(("rank 400 of 1300x1000", F.astype(np.uint32)))
    for i, (tag, A) in enumerate(cases):
        R, L, P, r, d = cuda.echelon_reduced_transform(p, A.copy())
        R2, r2, d2 = cuda.echelonize(p, A.copy(), reduced=True, unit_pivots=True)
        assert (r, d) == (r2, d2), tag
        assert np.array_equal(R, R2), tag
        _, P2, _, r3, _ = cuda.pluq(p, A.copy())
        assert P == P2[::-1] and r3 == r, tag
        _project_check(p, A, R, L, P, r, i)


@pytest.mark.gpu
def test_transform_device_views(cuda):
    """The device form on strided views: A a column slice of a wider
    buffer, L with a row stride larger than m; the columns and rows around
    them are left as they were."""
    import torch
    p = 65521
    m, n = 300, 410
    A = _kind(gen.dense_zp(41, m, n, p), p, 2, 42)
    want = oracle.echelon_reduced_L_zp(p, A)
    big = torch.full((m, n + 37), 7, dtype=torch.int32, device="cuda")
    big[:, 5:5 + n] = torch.from_numpy(A.view(np.int32))
    Lbig = torch.full((m, m + 19), 9, dtype=torch.int32, device="cuda")
    Av, Lv = big[:, 5:5 + n], Lbig[:, 3:3 + m]
    _, _, P, r, d = cuda.echelon_reduced_transform(p, Av, Lv)
    torch.cuda.synchronize()
    assert (r, d) == (want[3], want[4]) and P == want[2]
    assert np.array_equal(Av.cpu().numpy().view(np.uint32), want[0])
    assert np.array_equal(Lv.cpu().numpy().view(np.uint32), want[1])
    assert (big[:, :5] == 7).all() and (big[:, 5 + n:] == 7).all()
    assert (Lbig[:, :3] == 9).all() and (Lbig[:, 3 + m:] == 9).all()


@pytest.mark.gpu
def test_transform_host_strides(cuda):
    """Host arrays with row strides larger than the rows."""
    p = 251
    m, n = 90, 140
    A = gen.dense_zp(51, m, n, p)
    want = oracle.echelon_reduced_L_zp(p, A)
    Abig = np.full((m, n + 11), 3, dtype=np.uint32)
    Abig[:, :n] = A
    Lbig = np.full((m, m + 6), 5, dtype=np.uint32)
    R, L, P, r, d = cuda.echelon_reduced_transform(p, Abig[:, :n], Lbig[:, :m])
    assert (r, d) == (want[3], want[4]) and P == want[2]
    assert np.array_equal(Abig[:, :n], want[0]) and np.array_equal(Lbig[:, :m], want[1])
    assert (Abig[:, n:] == 3).all() and (Lbig[:, m:] == 5).all()

