"""PLUQ decomposition on the GPU against LELA's Elimination::pluq
(lela/algorithms/elimination.tcc:266-370): the golden fixtures computed by
LELA itself and the oracle's restatement, bit-exact in L and U, both
transposition lists, rank and det -- the counterpart of the PLUQ half of
tests/test-elimination.C.  Sizes cover several 64-column panels, blocks of
eight panels with delayed updates (more than 512 rows below the pivots),
pivots far below the current row, rank-deficient inputs, zero columns,
and moduli whose pivots LELA cannot invert."""
import numpy as np
import pytest

import golden_io
import oracle
from lela_b200 import gen, LELAError


def _check(cuda, p, A, tag):
    try:
        want = oracle.pluq_zp(p, A)
    except ArithmeticError:
        want = None
    if want is None:
        with pytest.raises(LELAError):
            cuda.pluq(p, A.copy())
        return
    got, gP, gQ, gr, gd = cuda.pluq(p, A.copy())
    assert (gr, gd) == (want[3], want[4]), tag
    assert gP == want[1], tag
    assert gQ == want[2], tag
    assert np.array_equal(got, want[0]), tag


@pytest.mark.gpu
def test_pluq_golden(cuda):
    for pre, p, st, r, d, A, E, P, Q in golden_io.pluq_cases():
        if st:
            with pytest.raises(LELAError):
                cuda.pluq(p, A.copy())
            continue
        got, gP, gQ, gr, gd = cuda.pluq(p, A.copy())
        assert (gr, gd) == (r, d), pre
        assert gP == P and gQ == Q, pre
        assert np.array_equal(got, E), pre


@pytest.mark.gpu
@pytest.mark.parametrize("p", [3, 251, 65521, 65536, 2147483647, 4294967291])
def test_pluq_against_oracle(cuda, p):
    rng = np.random.default_rng(p % 997)
    for (m, n) in ((1, 1), (7, 13), (13, 7), (70, 130), (130, 70), (300, 300), (700, 650)):
        for kind in range(4):
            A = gen.dense_zp(int(rng.integers(1 << 30)), m, n, p)
            if kind == 1:
                A[:, ::3] = 0
            elif kind == 2:
                r = max(1, min(m, n) // 3)
                F = (gen.dense_zp(1, m, r, p).astype(object) @ gen.dense_zp(2, r, n, p).astype(object)) % p
                A = F.astype(np.uint32)
            elif kind == 3:
                A[m // 2:] = 0
                A[:, :n // 2] = 0
            _check(cuda, p, A, (p, m, n, kind))


@pytest.mark.gpu
def test_pluq_blocks_and_far_pivots(cuda):
    """Delayed block updates (1600 rows: more than 512 below the first
    pivots) and the first panels' pivots far below the current row."""
    p = 65521
    A = gen.dense_zp(11, 1600, 1200, p)
    _check(cuda, p, A, "dense 1600x1200")
    B = gen.dense_zp(12, 1500, 900, p)
    B[:1100, :70] = 0
    _check(cuda, p, B, "far pivots")
    C = gen.dense_zp(13, 900, 1400, p)
    C[:, 200:330] = 0
    _check(cuda, p, C, "zero column band")


@pytest.mark.gpu
def test_pluq_device_path(cuda):
    import torch
    p = 2147483647
    A = gen.dense_zp(21, 520, 610, p)
    want = oracle.pluq_zp(p, A)
    T = torch.from_numpy(A.view(np.int32).copy()).cuda()
    got, gP, gQ, gr, gd = cuda.pluq(p, T)
    torch.cuda.synchronize()
    assert (gr, gd) == (want[3], want[4]) and gP == want[1] and gQ == want[2]
    assert np.array_equal(got.cpu().numpy().view(np.uint32), want[0])
