"""Z/p gemm and trsm over the other element types of Modular<T>: uint8,
uint16, float and double -- the element types of
tests/test-blas-zp-module.C:161-168 with its moduli, plus an even modulus
for the symmetric-range types.

* CPU: the restatement (oracle.gemm_zp_elem / trsm_zp_elem) against the
  fixtures LELA computed (tests/golden/make_elem_golden.py), bit-exact for
  odd moduli; for an even p the reference stores the residue p/2 as +p/2 or
  -p/2 depending on the path (ModularTraits<float>::reduce, lela/ring/
  modular.h:257-262), so there the residues agree and the restatement's
  representative is +p/2.
* GPU (through the C ABI, host and device pointers): bit-exact against the
  restatement, DiagonalEntryNotInvertible with LELA's index, the modulus
  bounds of ModularTraits<T>::valid_modulus, and one 2048^3 double gemm by
  Freivalds projections.
"""
import os

import numpy as np
import pytest

import oracle
import props
from lela_b200 import gen, DiagonalEntryNotInvertible, PreconditionFailed

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden", "elem_golden.npz")


def _gold():
    return np.load(GOLD)


def _cases(z, kind):
    pres = sorted({k[:k.rindex("_") + 1] for k in z.files if k.startswith(kind + "_")})
    return pres


def _same(p, want, got):
    """Bit-exact for odd p; for even p equal residues, with +p/2 on our side."""
    if p % 2:
        return want.dtype == got.dtype and np.array_equal(want, got)
    return np.array_equal(oracle.to_residues(want, p), oracle.to_residues(got, p))


def _rep(R, p, dt):
    return oracle.from_residues(R, p, dt)


# ------------------------------------------------------------------ CPU
def test_restatement_against_lela_fixtures():
    z = _gold()
    n = 0
    for pre in _cases(z, "gemm"):
        p, a, b = (int(x) for x in z[pre + "meta"])
        got = oracle.gemm_zp_elem(p, z[pre + "A"], z[pre + "B"], z[pre + "C"], a, b)
        assert _same(p, z[pre + "R"], got), pre
        n += 1
    for pre in _cases(z, "trsm"):
        p, a, upper, unit, bad = (int(x) for x in z[pre + "meta"])
        got, gbad = oracle.trsm_zp_elem(p, z[pre + "A"], z[pre + "B"], upper, unit, a)
        assert (gbad if gbad is not None else -1) == bad, pre
        if bad < 0:
            assert _same(p, z[pre + "R"], got), pre
        n += 1
    assert n == 8 * 3 + 8 * 6


def test_restatement_representation():
    """Residues to elements and back: symmetric range for float / double."""
    R = np.arange(7, dtype=np.uint32)
    assert oracle.from_residues(R, 7, np.float32).tolist() == [0, 1, 2, 3, -3, -2, -1]
    assert oracle.from_residues(R[:6], 6, np.float64).tolist() == [0, 1, 2, 3, -2, -1]
    assert oracle.from_residues(R, 7, np.uint8).tolist() == list(range(7))
    X = np.array([-3, -1, 0, 2, 3], dtype=np.float64)
    assert oracle.to_residues(X, 7).tolist() == [4, 6, 0, 2, 3]


# ------------------------------------------------------------------ GPU
TYPES = [(np.uint8, 251), (np.uint8, 2), (np.uint16, 65521), (np.uint16, 256),
         (np.float32, 2039), (np.float32, 4093), (np.float32, 10),
         (np.float64, 33554393), (np.float64, 67108859), (np.float64, 1000)]


@pytest.mark.gpu
def test_gemm_against_fixtures(cuda):
    z = _gold()
    for pre in _cases(z, "gemm"):
        p, a, b = (int(x) for x in z[pre + "meta"])
        C = z[pre + "C"].copy()
        got = cuda.gemm(p, a, z[pre + "A"], z[pre + "B"], b, C)
        assert got.dtype == z[pre + "R"].dtype
        assert _same(p, z[pre + "R"], got), pre
        if p % 2 == 0 and got.dtype.kind == "f":
            assert np.array_equal(got, _rep(oracle.to_residues(got, p), p, got.dtype))


@pytest.mark.gpu
@pytest.mark.parametrize("dt,p", TYPES)
def test_gemm_against_oracle(cuda, dt, p):
    """Host pointers, several shapes and coefficient patterns (tensor-core
    and small-K kernels both reached), one strided C."""
    for i, (m, n, k, a, b) in enumerate([(300, 257, 129, 1, 1), (64, 700, 1000, p - 1, 1),
                                         (513, 65, 33, 3 % p, 0), (1, 1, 1, 1, 1),
                                         (200, 200, 0, 1, 2 % p)]):
        A = _rep(gen.dense_zp(10 + i, m, k, p), p, dt)
        B = _rep(gen.dense_zp(20 + i, k, n, p), p, dt)
        C = _rep(gen.dense_zp(30 + i, m, n, p), p, dt)
        want = oracle.gemm_zp_elem(p, A, B, C, a, b)
        got = cuda.gemm(p, a, A, B, b, C.copy())
        assert np.array_equal(got, want), (dt, p, i)
    # strided C: a column slice of a wider array
    A = _rep(gen.dense_zp(40, 100, 80, p), p, dt)
    B = _rep(gen.dense_zp(41, 80, 60, p), p, dt)
    W = _rep(gen.dense_zp(42, 100, 75, p), p, dt)
    want = oracle.gemm_zp_elem(p, A, B, W[:, 5:65], 1, 1)
    before = W.copy()
    cuda.gemm(p, 1, A, B, 1, W[:, 5:65])
    assert np.array_equal(W[:, 5:65], want)
    assert np.array_equal(W[:, :5], before[:, :5]) and np.array_equal(W[:, 65:], before[:, 65:])


@pytest.mark.gpu
@pytest.mark.parametrize("dt,p", [(np.uint8, 251), (np.uint16, 65521), (np.float32, 4093),
                                  (np.float64, 67108859)])
def test_gemm_device_pointers(cuda, dt, p):
    import torch
    m, n, k = 777, 300, 1500
    A = _rep(gen.dense_zp(50, m, k, p), p, dt)
    B = _rep(gen.dense_zp(51, k, n, p), p, dt)
    C = _rep(gen.dense_zp(52, m, n, p), p, dt)
    want = oracle.gemm_zp_elem(p, A, B, C, p - 2, 5)
    dev = lambda X: torch.from_numpy(X.view(np.int16) if dt == np.uint16 else X).cuda()
    dC = dev(C)
    cuda.gemm(p, p - 2, dev(A), dev(B), 5, dC)
    torch.cuda.synchronize()
    got = dC.cpu().numpy()
    if dt == np.uint16:
        got = got.view(np.uint16)
    assert np.array_equal(got, want)


@pytest.mark.gpu
def test_trsm_against_fixtures(cuda):
    z = _gold()
    for pre in _cases(z, "trsm"):
        p, a, upper, unit, bad = (int(x) for x in z[pre + "meta"])
        B = z[pre + "B"].copy()
        if bad >= 0:
            with pytest.raises(DiagonalEntryNotInvertible) as e:
                cuda.trsm(p, a, z[pre + "A"], B, upper, unit)
            assert e.value.idx == bad, pre
            assert np.array_equal(B, z[pre + "B"]), pre  # unchanged
            continue
        got = cuda.trsm(p, a, z[pre + "A"], B, upper, unit)
        assert _same(p, z[pre + "R"], got), pre


@pytest.mark.gpu
@pytest.mark.parametrize("dt,p", TYPES)
def test_trsm_against_oracle(cuda, dt, p):
    """Both triangles, unit and general diagonals, sizes across the
    block-substitution and inverse-leaf solvers."""
    for i, (m, n) in enumerate([(7, 3), (300, 70), (1100, 40)]):
        for upper in (0, 1):
            for unit in (0, 1):
                L = gen.dense_zp(60 + i, m, m, p)
                L = np.triu(L) if upper else np.tril(L)
                if unit:
                    np.fill_diagonal(L, 1)
                else:
                    d = np.diag(L).copy()
                    d[d == 0] = 1
                    if p % 2 == 0:
                        d[d % 2 == 0] += 1  # odd entries are units when p is a power of two
                    np.fill_diagonal(L, d % p)
                A = _rep(L, p, dt)
                B = _rep(gen.dense_zp(70 + i, m, n, p), p, dt)
                want, wbad = oracle.trsm_zp_elem(p, A, B, upper, unit, 5 % p)
                if wbad is not None:
                    with pytest.raises(DiagonalEntryNotInvertible) as e:
                        cuda.trsm(p, 5 % p, A, B.copy(), upper, unit)
                    assert e.value.idx == wbad
                    continue
                got = cuda.trsm(p, 5 % p, A, B.copy(), upper, unit)
                assert np.array_equal(got, want), (dt, p, m, upper, unit)


@pytest.mark.gpu
def test_modulus_bounds(cuda):
    """ModularTraits<T>::valid_modulus: p < 2^8, 2^16, 4096, 2^26."""
    for dt, p in [(np.uint8, 256), (np.uint16, 65536), (np.float32, 4096), (np.float64, 1 << 26)]:
        A = np.zeros((4, 4), dtype=dt)
        with pytest.raises(PreconditionFailed):
            cuda.gemm(p, 1, A, A, 1, A.copy())
        with pytest.raises(PreconditionFailed):
            cuda.trsm(p, 1, A + 1, A.copy(), True, True)


@pytest.mark.gpu
def test_gemm_double_2048(cuda):
    """2048^3 over Modular<double> at p = 67108859 (four limbs), checked by
    Freivalds projections on the residues."""
    p, n = 67108859, 2048
    A = _rep(gen.dense_zp(80, n, n, p), p, np.float64)
    B = _rep(gen.dense_zp(81, n, n, p), p, np.float64)
    C = _rep(gen.dense_zp(82, n, n, p), p, np.float64)
    got = cuda.gemm(p, 3, A, B, p - 1, C.copy())
    r = lambda X: oracle.to_residues(X, p)
    assert props.freivalds_gemm(p, r(A), r(B), r(C), r(got), 3, p - 1)
    assert np.abs(got).max() <= p // 2
