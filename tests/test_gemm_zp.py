"""Z/p gemm on the GPU against the CPU oracle -- the CUDAModule counterpart
of LELA's module-consistency tests (tests/test-blas-level3.h:1376-1461,
testgemmConsistency: the same gemm under two contexts, compared with
BLAS3::equal).  Integer results must be bit-identical."""
import numpy as np
import pytest

import oracle
from lela_b200 import gen, api

import props

P_CASES = [2, 251, 256, 257, 65521, 65536, 65537, 268435455, 268435457, 2147483647, 4294967291]
SHAPES = [(1, 1, 1), (17, 33, 5), (128, 128, 128), (130, 257, 300), (64, 300, 1000)]
COEFFS = [(1, 1), ("m1", 1), (3, 0), (0, 5), (7, 11)]


def _coef(x, p):
    return (p - 1) if x == "m1" else x % p


@pytest.mark.gpu
@pytest.mark.parametrize("kernel", [api.GEMM_TC, api.GEMM_PLAIN, api.GEMM_SMALLK, api.GEMM_AUTO])
@pytest.mark.parametrize("p", P_CASES)
def test_gemm_shapes_moduli(cuda, kernel, p):
    cuda.set_gemm_kernel(kernel)
    try:
        for si, (m, n, k) in enumerate(SHAPES):
            for ci, (a, b) in enumerate(COEFFS):
                a, b = _coef(a, p), _coef(b, p)
                seed = 1000 * si + 10 * ci + p % 97
                A = gen.dense_zp(seed, m, k, p)
                B = gen.dense_zp(seed + 1, k, n, p)
                C = gen.dense_zp(seed + 2, m, n, p)
                want = oracle.gemm_zp(p, A, B, C, a, b)
                got = cuda.gemm(p, a, A, B, b, C.copy())
                assert np.array_equal(got, want), (kernel, p, m, n, k, a, b)
    finally:
        cuda.set_gemm_kernel(api.GEMM_AUTO)


@pytest.mark.gpu
def test_gemm_config0_512(cuda):
    """The plain 512^3 case: p = 65521, C <- A*B + C, entries uniform in
    [0, p), seed 0; both GPU kernels against the oracle."""
    p, n = 65521, 512
    A = gen.dense_zp(0, n, n, p)
    B = gen.dense_zp(1, n, n, p)
    C = gen.dense_zp(2, n, n, p)
    want = oracle.gemm_zp(p, A, B, C, 1, 1, threads=8)
    for kernel in (api.GEMM_TC, api.GEMM_PLAIN):
        cuda.set_gemm_kernel(kernel)
        got = cuda.gemm(p, 1, A, B, 1, C.copy())
        assert np.array_equal(got, want), kernel
    cuda.set_gemm_kernel(api.GEMM_AUTO)


@pytest.mark.gpu
def test_gemm_strided_views(cuda):
    """Submatrix views keep the parent's row stride (lela/matrix/dense.h:
    425-429); the C ABI takes it as the leading dimension."""
    p = 65521
    big = gen.dense_zp(5, 300, 400, p)
    A = big[10:110, 20:90]     # 100 x 70, lda = 400
    B = big[120:190, 3:203]    # 70 x 200
    Cbig = gen.dense_zp(6, 150, 260, p)
    C = Cbig[7:107, 30:230]    # 100 x 200, ldc = 260
    want = oracle.gemm_zp(p, A, B, C, 5, 3)
    before = Cbig.copy()
    cuda.gemm(p, 5, A, B, 3, C)
    assert np.array_equal(C, want)
    mask = np.ones_like(Cbig, dtype=bool)
    mask[7:107, 30:230] = False
    assert np.array_equal(Cbig[mask], before[mask])


@pytest.mark.gpu
def test_gemm_k_chunking(cuda):
    """K above the 32768-term overflow bound of one tensor-core pass."""
    p = 65521
    m, n, k = 40, 72, 40000
    A = np.full((m, k), p - 1, dtype=np.uint32)   # worst case limbs 0xF0, 0xFF
    A[:, ::3] = gen.dense_zp(8, m, k, p)[:, ::3]
    B = np.full((k, n), p - 1, dtype=np.uint32)
    C = gen.dense_zp(9, m, n, p)
    want = oracle.gemm_zp(p, A, B, C, 1, 1, threads=8)
    got = cuda.gemm(p, 1, A, B, 1, C.copy())
    assert np.array_equal(got, want)


@pytest.mark.gpu
def test_gemm_max_entries(cuda):
    """All entries p-1: the largest limb products and accumulator values."""
    for p in (251, 65521, 4294967291):
        A = np.full((200, 33000), p - 1, dtype=np.uint32)
        B = np.full((33000, 130), p - 1, dtype=np.uint32)
        C = np.full((200, 130), p - 1, dtype=np.uint32)
        want = oracle.gemm_zp(p, A[:, :33000], B, C, p - 1, p - 1, threads=8)
        got = cuda.gemm(p, p - 1, A, B, p - 1, C.copy())
        assert np.array_equal(got, want), p


@pytest.mark.gpu
def test_gemm_device_tensors(cuda):
    """The _dev entry point on torch CUDA tensors, on the caller's stream."""
    import torch
    p = 2147483647
    m, n, k = 300, 200, 500
    A = gen.dense_zp(11, m, k, p)
    B = gen.dense_zp(12, k, n, p)
    C = gen.dense_zp(13, m, n, p)
    want = oracle.gemm_zp(p, A, B, C, 2, 3)
    dev = lambda x: torch.from_numpy(x.view(np.int32)).cuda()
    dA, dB, dC = dev(A), dev(B), dev(C)
    s = torch.cuda.Stream()
    cuda.set_stream(s)
    try:
        cuda.gemm(p, 2, dA, dB, 3, dC)
        cuda.synchronize()
    finally:
        cuda.set_stream(None)
    got = dC.cpu().numpy().view(np.uint32)
    assert np.array_equal(got, want)


@pytest.mark.gpu
def test_gemm_8192_property(cuda):
    """Full-size workload (8192^3, p = 65521): Freivalds certificate."""
    p, n = 65521, 8192
    A = gen.dense_zp(21, n, n, p)
    B = gen.dense_zp(22, n, n, p)
    C0 = gen.dense_zp(23, n, n, p)
    C = cuda.gemm(p, 1, A, B, 1, C0.copy())
    assert props.freivalds_gemm(p, A, B, C0, C, 1, 1)


@pytest.mark.gpu
@pytest.mark.parametrize("p", [251, 65521, 2147483647])
def test_gemm_host_row_blocks(cuda, p):
    """Host-pointer gemms large enough for the row-block pipeline (copies on
    two streams overlapped with the per-block products): ragged last
    block, row strides larger than the rows, b = 0 (C never read) and
    b != 0, one limb count per modulus."""
    big = gen.dense_zp(31, 1300, 700, p)
    A = big[3:1203, 10:310]                   # 1200 x 300, lda = 700
    B = gen.dense_zp(32, 300, 520, p)
    Cbig = gen.dense_zp(33, 1250, 600, p)
    C = Cbig[20:1220, 40:560]                 # 1200 x 520, ldc = 600
    for a, b in ((1, 1), (p - 1, 0), (7, 11)):
        want = oracle.gemm_zp(p, A, B, C, a, b, threads=8)
        before = Cbig.copy()
        cuda.gemm(p, a, A, B, b, C)
        assert np.array_equal(C, want), (p, a, b)
        mask = np.ones_like(Cbig, dtype=bool)
        mask[20:1220, 40:560] = False
        assert np.array_equal(Cbig[mask], before[mask])
        C[...] = want                         # next case starts from this C


@pytest.mark.gpu
@pytest.mark.parametrize("tile", [api.GEMM_TILE_WIDE, api.GEMM_TILE_DOUBLE])
@pytest.mark.parametrize("p", [251, 65521, 2147483647])
def test_gemm_tile_variants(cuda, tile, p):
    """Both tensor-core tile variants (one accumulator buffer / two) on
    ragged shapes, every epilogue mode (C += AB, C -= AB, C = aAB,
    aAB + bC), and device matrices whose row strides and column offsets
    are not multiples of four entries (the epilogue's 16-byte loads and
    stores fall back to single entries there)."""
    import torch
    cuda.set_gemm_kernel(api.GEMM_TC)
    cuda.set_gemm_tile(tile)
    dev = lambda x: torch.from_numpy(np.ascontiguousarray(x).view(np.int32)).cuda()
    try:
        for si, (m, n, k) in enumerate([(130, 257, 300), (300, 130, 40), (257, 515, 2100),
                                        (129, 67, 5)]):
            A = gen.dense_zp(70 + si, m, k, p)
            B = gen.dense_zp(80 + si, k, n, p)
            for ci, (a, b) in enumerate([(1, 1), (p - 1, 1), (3, 0), (7, 11)]):
                C = gen.dense_zp(90 + 10 * si + ci, m, n, p)
                want = oracle.gemm_zp(p, A, B, C, a, b)
                got = cuda.gemm(p, a, A, B, b, C.copy())
                assert np.array_equal(got, want), (tile, p, m, n, k, a, b, "host")
                # device: C a view at column 1 of a wider matrix (stride n + 3)
                W = np.zeros((m, n + 3), dtype=np.uint32)
                W[:, 1:n + 1] = C
                dW = dev(W)
                cuda.gemm(p, a, dev(A), dev(B), b, dW[:, 1:n + 1])
                cuda.synchronize()
                gw = dW.cpu().numpy().view(np.uint32)
                assert np.array_equal(gw[:, 1:n + 1], want), (tile, p, m, n, k, a, b, "view")
                assert not gw[:, 0].any() and not gw[:, n + 1:].any()
    finally:
        cuda.set_gemm_kernel(api.GEMM_AUTO)
        cuda.set_gemm_tile(api.GEMM_TILE_AUTO)
