"""Z/p trsm on the GPU against the oracle and LELA's golden results -- the
counterpart of testtrsmConsistency (tests/test-blas-level3.h:1538-1604) and
of the trsm/trmm round trips (testTrsmLower/Upper, :715/:778)."""
import numpy as np
import pytest

import golden_io
import oracle
from lela_b200 import gen, DiagonalEntryNotInvertible
from lela_b200.api import TRSM_AUTO, TRSM_BLOCKS, TRSM_INVERSE

import props


@pytest.mark.gpu
def test_trsm_golden(cuda):
    for pre, p, upper, unit, a, bad, A, B, R in golden_io.trsm_cases():
        if bad is None:
            got = cuda.trsm(p, a, A, B.copy(), upper, unit)
            assert np.array_equal(got, R), pre
        else:
            with pytest.raises(DiagonalEntryNotInvertible) as ei:
                cuda.trsm(p, a, A, B.copy(), upper, unit)
            assert ei.value.idx == bad, pre


@pytest.mark.gpu
@pytest.mark.parametrize("p", [251, 65521, 2147483647])
def test_trsm_against_oracle(cuda, p):
    rng = np.random.default_rng(p % 1000)
    for m, n in [(1, 1), (5, 3), (64, 10), (65, 7), (130, 33), (300, 200), (513, 64)]:
        for upper in (0, 1):
            for unit in (0, 1):
                U = gen.upper_zp(m * 7 + n, m, p, unit=bool(unit))
                A = U if upper else np.ascontiguousarray(U.T)
                B = gen.dense_zp(m + n, m, n, p)
                a = int(rng.integers(1, p))
                want, _ = oracle.trsm_zp(p, A, B, upper, unit, a)
                got = cuda.trsm(p, a, A, B.copy(), upper, unit)
                assert np.array_equal(got, want), (p, m, n, upper, unit)


@pytest.mark.gpu
def test_trsm_alpha_zero_and_singular(cuda):
    p = 65521
    U = gen.upper_zp(3, 200, p)
    U[17, 17] = 0
    U[150, 150] = 0
    B = gen.dense_zp(4, 200, 9, p)
    # a = 0: B <- 0 without looking at A (lela/blas/level3-generic.tcc:433-434)
    got = cuda.trsm(p, 0, U, B.copy(), 1, 0)
    assert not got.any()
    with pytest.raises(DiagonalEntryNotInvertible) as ei:
        cuda.trsm(p, 1, U, B.copy(), 1, 0)
    assert ei.value.idx == 150
    with pytest.raises(DiagonalEntryNotInvertible) as ei:
        cuda.trsm(p, 1, np.ascontiguousarray(U.T), B.copy(), 0, 0)
    assert ei.value.idx == 17
    # p >= 2^31: LELA's 32-bit Euclid cannot invert; the same index is reported
    want = oracle.trsm_zp(4294967291, U, B, 1, 0, 1)[1]
    with pytest.raises(DiagonalEntryNotInvertible) as ei:
        cuda.trsm(4294967291, 1, U, B.copy(), 1, 0)
    assert ei.value.idx == want


@pytest.mark.gpu
@pytest.mark.parametrize("kernel", [TRSM_BLOCKS, TRSM_INVERSE])
def test_trsm_8192_unit_lower_property(cuda, kernel):
    """The full trsm workload (8192 x 8192 unit-lower L, 8192 x 4096 RHS,
    p = 65521): L * X == B checked by random projection (Freivalds)."""
    p, m, n = 65521, 8192, 4096
    L = gen.unit_lower_zp(31, m, p)
    B = gen.dense_zp(32, m, n, p)
    cuda.set_trsm_kernel(kernel)
    try:
        X = cuda.trsm(p, 1, L, B.copy(), 0, 1)
    finally:
        cuda.set_trsm_kernel(TRSM_AUTO)
    zero = np.zeros_like(B)
    # L X + 0 == B  <=>  gemm(L, X) reproduces B
    assert props.freivalds_gemm(p, L, X, zero, B, 1, 0)


@pytest.mark.gpu
@pytest.mark.parametrize("kernel", [TRSM_BLOCKS, TRSM_INVERSE])
@pytest.mark.parametrize("p", [251, 65521, 2147483647, 4294967291, 1000000])
def test_trsm_kernels_against_oracle(cuda, kernel, p):
    """Both diagonal-block solvers (256-row substitution, 512-row inverses
    applied on the tensor cores) give the oracle's B: sizes around the block
    and leaf boundaries, narrow and wide right-hand sides, alpha != 1, and
    moduli whose diagonal inverses need a unit diagonal (p >= 2^31, where
    LELA's inversion fails, and the composite 10^6)."""
    rng = np.random.default_rng(p % 997 + kernel)
    only_unit = p >= 2**31 or p == 1000000
    cuda.set_trsm_kernel(kernel)
    try:
        for m, n in [(63, 5), (65, 300), (257, 40), (513, 300), (700, 1), (1100, 260), (1537, 97)]:
            for upper in (0, 1):
                for unit in ((1,) if only_unit else (0, 1)):
                    U = gen.upper_zp(m * 3 + n + upper, m, p, unit=bool(unit))
                    A = U if upper else np.ascontiguousarray(U.T)
                    B = gen.dense_zp(m + 2 * n, m, n, p)
                    a = int(rng.integers(1, p))
                    want, _ = oracle.trsm_zp(p, A, B, upper, unit, a)
                    got = cuda.trsm(p, a, A, B.copy(), upper, unit)
                    assert np.array_equal(got, want), (kernel, p, m, n, upper, unit)
    finally:
        cuda.set_trsm_kernel(TRSM_AUTO)


@pytest.mark.gpu
def test_trsm_inverse_singular(cuda):
    """The inverse leaves report LELA's index for a singular diagonal and
    leave B unchanged, like the substitution."""
    p = 65521
    U = gen.upper_zp(5, 1200, p)
    U[100, 100] = 0
    U[1000, 1000] = 0
    B = gen.dense_zp(6, 1200, 300, p)
    cuda.set_trsm_kernel(TRSM_INVERSE)
    try:
        for upper, want in ((1, 1000), (0, 100)):
            A = U if upper else np.ascontiguousarray(U.T)
            X = B.copy()
            with pytest.raises(DiagonalEntryNotInvertible) as ei:
                cuda.trsm(p, 1, A, X, upper, 0)
            assert ei.value.idx == want
            assert np.array_equal(X, B)
    finally:
        cuda.set_trsm_kernel(TRSM_AUTO)
