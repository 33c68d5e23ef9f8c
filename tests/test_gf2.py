"""GF(2) gemm and echelon form on the GPU against LELA's generic GF(2) path
(the golden fixtures) and the oracle: the counterpart of
tests/test-blas-generic-module-gf2.C and the GF(2) half of
tests/test-gauss-jordan.C / test-elimination.C.  Bit-exact."""
import numpy as np
import pytest

import golden_io
import oracle
from lela_b200 import gen

KERNELS = (1, 2)  # int8-expanded tensor cores, four-Russians


@pytest.mark.gpu
@pytest.mark.parametrize("kernel", KERNELS)
def test_gf2_gemm_golden(cuda, kernel):
    cuda.set_gf2_kernel(kernel)
    try:
        for pre, m, n, k, A, B, C, R in golden_io.gf2_gemm_cases():
            got = cuda.gemm_gf2(A, B, C.copy(), n, k, 1, 1)
            assert np.array_equal(got, R), (kernel, pre)
    finally:
        cuda.set_gf2_kernel(0)


@pytest.mark.gpu
@pytest.mark.parametrize("kernel", KERNELS)
def test_gf2_gemm_against_oracle(cuda, kernel):
    cuda.set_gf2_kernel(kernel)
    try:
        for seed, (m, n, k) in enumerate([(1, 1, 1), (7, 65, 63), (130, 257, 300), (300, 64, 1000),
                                          (512, 600, 2100), (129, 1000, 64)]):
            A = gen.dense_gf2(seed, m, k)
            B = gen.dense_gf2(seed + 100, k, n)
            C = gen.dense_gf2(seed + 200, m, n)
            for a, b in ((1, 1), (1, 0), (0, 1)):
                want = oracle.gemm_gf2(A, B, C, k, n, a, b)
                got = cuda.gemm_gf2(A, B, C.copy(), n, k, a, b)
                assert np.array_equal(got, want), (kernel, m, n, k, a, b)
    finally:
        cuda.set_gf2_kernel(0)


@pytest.mark.gpu
def test_gf2_gemm_kernels_agree_large(cuda):
    """4096^3: the two kernels give the same product (and so LELA's, by the
    tests above); Freivalds-style check on random vectors as well."""
    n = 4096
    A = gen.dense_gf2(1, n, n)
    B = gen.dense_gf2(2, n, n)
    C0 = np.zeros((n, n // 64), dtype=np.uint64)
    outs = []
    for kernel in KERNELS:
        cuda.set_gf2_kernel(kernel)
        outs.append(cuda.gemm_gf2(A, B, C0.copy(), n, n, 1, 0))
    cuda.set_gf2_kernel(0)
    assert np.array_equal(outs[0], outs[1])
    a = gen.unpack_gf2(A, n).astype(np.int64)
    b = gen.unpack_gf2(B, n).astype(np.int64)
    c = gen.unpack_gf2(outs[0], n).astype(np.int64)
    x = np.random.default_rng(0).integers(0, 2, size=n)
    assert np.array_equal((c @ x) % 2, (a @ ((b @ x) % 2)) % 2)


@pytest.mark.gpu
def test_gf2_echelon_golden(cuda):
    for pre, m, n, r, A, E in golden_io.gf2_echelon_cases():
        got, gr = cuda.echelonize_gf2(A.copy(), n)
        assert gr == r, pre
        assert np.array_equal(got, E), pre


@pytest.mark.gpu
def test_gf2_echelon_against_oracle(cuda):
    for seed, (m, n, r) in enumerate([(1, 1, 1), (5, 70, 5), (64, 64, 64), (100, 90, 40),
                                      (300, 200, 150), (257, 513, 200), (700, 700, 650)]):
        A = gen.planted_rank_gf2(seed, m, n, r)
        if seed % 2:
            A[:, 0] = 0  # a zero first word column
        want, wr = oracle.echelon_gf2(A, n)
        got, gr = cuda.echelonize_gf2(A.copy(), n)
        assert gr == wr, (m, n, r)
        assert np.array_equal(got, want), (m, n, r)
    for seed, (m, n) in enumerate([(200, 300), (333, 129)]):
        A = gen.dense_gf2(50 + seed, m, n)
        want, wr = oracle.echelon_gf2(A, n)
        got, gr = cuda.echelonize_gf2(A.copy(), n)
        assert gr == wr and np.array_equal(got, want), (m, n)


@pytest.mark.gpu
def test_gf2_echelon_pivots_far_below(cuda):
    """The first 4500 rows are zero in the leading columns, so pivots come
    from rows beyond the block the search keeps on chip."""
    m, n = 6000, 200
    A = gen.dense_gf2(77, m, n)
    A[:4500, 0] &= ~np.uint64((1 << 40) - 1)
    A[4500:5200, 0] &= ~np.uint64(0xFFF)
    want, wr = oracle.echelon_gf2(A, n)
    got, gr = cuda.echelonize_gf2(A.copy(), n)
    assert gr == wr
    assert np.array_equal(got, want)


@pytest.mark.gpu
def test_gf2_echelon_blocks(cuda):
    """Several blocks of four word-panels with delayed trailing updates
    (many rows below the pivots), rank-deficient and dense inputs, a band of
    zero columns and pivots far below in the first block."""
    for seed, (m, n, r) in enumerate([(1500, 1300, 1100), (1200, 2000, 1200), (2100, 700, 650)]):
        A = gen.planted_rank_gf2(90 + seed, m, n, r)
        if seed == 1:
            A[:, 5] = 0                                   # a whole word column without pivots
        want, wr = oracle.echelon_gf2(A, n)
        got, gr = cuda.echelonize_gf2(A.copy(), n)
        assert gr == wr, (m, n, r)
        assert np.array_equal(got, want), (m, n, r)
    m, n = 2500, 900
    A = gen.dense_gf2(93, m, n)
    A[:1800, :2] = 0                                      # the first panels' pivots far below
    want, wr = oracle.echelon_gf2(A, n)
    got, gr = cuda.echelonize_gf2(A.copy(), n)
    assert gr == wr and np.array_equal(got, want)


@pytest.mark.gpu
@pytest.mark.parametrize("kernel", KERNELS)
def test_gf2_gemm_strided_c_keeps_neighbour_bits(cuda, kernel):
    """C is the first 100 columns of a 256-column matrix (row stride 4
    words): the product lands in bits 0..99, and bits 100..255 of every row
    -- the rest of the last word and the two words after it -- keep their
    values, whatever b is.  Host and device paths."""
    import torch
    m, n, k = 150, 100, 333
    A = gen.dense_gf2(5, m, k)
    B = gen.dense_gf2(6, k, n)
    W = gen.dense_gf2(7, m, 256)
    cuda.set_gf2_kernel(kernel)
    try:
        for a, b in ((1, 1), (1, 0), (0, 0)):
            Cn = np.ascontiguousarray(W[:, :2])
            Cn[:, 1] &= np.uint64((1 << 36) - 1)          # columns 0..99 only
            want = oracle.gemm_gf2(A, B, Cn, k, n, a, b)
            tail = ~np.uint64((1 << 36) - 1)
            want[:, 1] |= W[:, 1] & tail
            for dev in (False, True):
                Wc = W.copy()
                if dev:
                    Wt = torch.from_numpy(Wc.view(np.int64)).cuda()
                    cuda.gemm_gf2(torch.from_numpy(A.view(np.int64)).cuda(),
                                  torch.from_numpy(B.view(np.int64)).cuda(), Wt[:, :2], n, k, a, b)
                    torch.cuda.synchronize()
                    Wc = Wt.cpu().numpy().view(np.uint64)
                else:
                    cuda.gemm_gf2(A, B, Wc[:, :2], n, k, a, b)
                assert np.array_equal(Wc[:, :2], want), (kernel, a, b, dev)
                assert np.array_equal(Wc[:, 2:], W[:, 2:]), (kernel, a, b, dev)
    finally:
        cuda.set_gf2_kernel(0)


@pytest.mark.gpu
def test_gf2_gemm_host_row_blocks(cuda):
    """The host-pointer GF(2) gemm of a large tensor-core shape works in row
    blocks with its copies overlapped: ragged blocks (1500 rows), a partial
    last word of C (700 columns: the bits past column 700 of a row of C are
    kept), b = 0 and 1, and host rows wider than the matrices (views of
    larger arrays)."""
    m, n, k = 1500, 700, 300
    nw, kw = (n + 63) // 64, (k + 63) // 64
    A = gen.dense_gf2(141, m, k)
    B = gen.dense_gf2(142, k, n)
    for b in (0, 1):
        W = gen.dense_gf2(143 + b, m, n + 128)  # C = its first nw words
        C = W[:, :nw]
        tail = np.uint64((1 << (n % 64)) - 1)
        C0 = C.copy()
        C0[:, -1] &= tail
        want = oracle.gemm_gf2(A, B, C0, k, n, 1, b)
        before = W.copy()
        Aw = np.zeros((m, kw + 3), dtype=np.uint64)
        Aw[:, :kw] = A
        cuda.gemm_gf2(Aw[:, :kw], B, C, n, k, 1, b)
        got = W[:, :nw]
        assert np.array_equal(got[:, :-1], want[:, :-1]), b
        assert np.array_equal(got[:, -1] & tail, want[:, -1] & tail), b
        assert np.array_equal(got[:, -1] & ~tail, before[:, nw - 1] & ~tail), b  # bits past n kept
        assert np.array_equal(W[:, nw:], before[:, nw:]), b
