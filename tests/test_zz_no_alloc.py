"""lela_cuda_gemm_zp_u32_noalloc: the Z/p tensor-core gemm for callers that
cannot allocate device memory (their device memory belongs to a host
framework's allocator or a fixed budget, or cudaMalloc's possible device
synchronisation is not allowed on their path).  The entry point keeps its
scratch in a fixed array inside the library; these tests call it through
the C ABI, two or more calls in a row sharing that scratch, and compare
every result with the regular device-pointer entry point
lela_cuda_gemm_zp_u32_dev and with the CPU oracle (bit-exact, as every Z/p
test here).  Covered: one, two and four limbs; K past one 32768-term chunk
(the scratch reused within a call, beta = 1 after the first chunk); leading
dimensions wider than the rows; a caller's stream; the k = 0 and a = 0
scale paths; the size limit.

The file name sorts last so that a run stopping at the first failure has
already run every other test; it also passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

import oracle
from lela_b200 import api, gen

_P = ctypes.c_void_p
_S = ctypes.c_size_t
_U = ctypes.c_uint32


def _noalloc_fn():
    fn = api.load_library().lela_cuda_gemm_zp_u32_noalloc
    fn.argtypes = [_S, _S, _S, _U, _U, _P, _S, _P, _S, _U, _P, _S, _P]
    fn.restype = ctypes.c_int
    return fn


def _dev(x, ld=None):
    """Device copy of a host uint32 matrix with row stride ld >= its width
    (the padding columns hold a marker value)."""
    import torch
    m, n = x.shape
    ld = ld or n
    buf = np.full((m, ld), 0x5A5A5A5A, dtype=np.uint32)
    buf[:, :n] = x
    return torch.from_numpy(buf.view(np.int32)).cuda()


def _host(t, n):
    return t.cpu().numpy().view(np.uint32)[:, :n]


@pytest.mark.gpu
def test_noalloc_matches_dev_entry_point_twice():
    import torch
    fn = _noalloc_fn()
    cm = api.CudaModule(0)
    cases = [(65521, 700, 650, 900, 3, 5), (2147483647, 300, 257, 1000, 1, 1),
             (251, 513, 129, 77, 250, 0)]
    try:
        for i, (p, m, n, k, a, b) in enumerate(cases):
            A = gen.dense_zp(500 + i, m, k, p)
            B = gen.dense_zp(600 + i, k, n, p)
            C = gen.dense_zp(700 + i, m, n, p)
            want = oracle.gemm_zp(p, A, B, C, a, b)
            dA, dB = _dev(A), _dev(B)
            ref_C, new_C = _dev(C), _dev(C)
            cm.gemm(p, a, dA, dB, b, ref_C)
            cm.synchronize()
            torch.cuda.synchronize()
            st = fn(m, n, k, p, a, dA.data_ptr(), k, dB.data_ptr(), n, b, new_C.data_ptr(), n, None)
            assert st == api.OK, st
            torch.cuda.synchronize()
            assert torch.equal(ref_C, new_C), "call %d differs from lela_cuda_gemm_zp_u32_dev" % i
            assert np.array_equal(_host(new_C, n), want), "call %d differs from the oracle" % i
    finally:
        cm.close()


@pytest.mark.gpu
def test_noalloc_k_chunks_strides_and_stream():
    """k = 40000 > 32768: two chunks through the same scratch in one call;
    lda, ldb, ldc wider than the rows (the padding must stay untouched); the
    work queued on a torch stream passed as the cudaStream_t; then a second
    call with other operands that must not see the first call's scratch."""
    import torch
    fn = _noalloc_fn()
    s = torch.cuda.Stream()
    cases = [(251, 256, 256, 40000, 1, 1, (40016, 272, 260)),
             (65521, 200, 333, 35000, 7, 2, (35001, 340, 333)),
             (4294967291, 96, 70, 33000, 5, 9, (33000, 70, 75))]
    for i, (p, m, n, k, a, b, (lda, ldb, ldc)) in enumerate(cases):
        A = gen.dense_zp(800 + i, m, k, p)
        B = gen.dense_zp(810 + i, k, n, p)
        C = gen.dense_zp(820 + i, m, n, p)
        want = oracle.gemm_zp(p, A, B, C, a, b, threads=8)
        dA, dB, dC = _dev(A, lda), _dev(B, ldb), _dev(C, ldc)
        torch.cuda.synchronize()
        st = fn(m, n, k, p, a, dA.data_ptr(), lda, dB.data_ptr(), ldb, b, dC.data_ptr(), ldc,
                ctypes.c_void_p(s.cuda_stream))
        assert st == api.OK, (i, st)
        torch.cuda.synchronize()
        got = dC.cpu().numpy().view(np.uint32)
        assert np.array_equal(got[:, :n], want), "case %d differs from the oracle" % i
        assert (got[:, n:] == 0x5A5A5A5A).all(), "case %d wrote past the rows of C" % i


@pytest.mark.gpu
def test_noalloc_scale_paths():
    """k = 0 and a = 0: C <- b*C (b = 3, then b = 0), no product."""
    import torch
    fn = _noalloc_fn()
    p, m, n, k = 65521, 129, 77, 50
    A = gen.dense_zp(900, m, k, p)
    B = gen.dense_zp(901, k, n, p)
    C = gen.dense_zp(902, m, n, p)
    for kk, a, b in ((k, 0, 3), (0, 5, 3), (k, 0, 0)):
        dA, dB, dC = _dev(A), _dev(B), _dev(C, n + 3)
        st = fn(m, n, kk, p, a, dA.data_ptr(), k, dB.data_ptr(), n, b, dC.data_ptr(), n + 3, None)
        assert st == api.OK, st
        torch.cuda.synchronize()
        got = dC.cpu().numpy().view(np.uint32)
        want = (C.astype(np.uint64) * b % p).astype(np.uint32)
        assert np.array_equal(got[:, :n], want), (kk, a, b)
        assert (got[:, n:] == 0x5A5A5A5A).all()


@pytest.mark.gpu
def test_noalloc_rejects_sizes_beyond_scratch():
    import torch
    fn = _noalloc_fn()
    x = torch.zeros(16, dtype=torch.int32, device="cuda")
    # 2 limbs * (20000 + 20000) rows * 4096 bytes > 64 MiB
    st = fn(20000, 20000, 4096, 65521, 1, x.data_ptr(), 4096, x.data_ptr(), 20000, 1,
            x.data_ptr(), 20000, None)
    assert st == api.ERR_ARG
    # leading dimension smaller than the row
    st = fn(16, 16, 16, 65521, 1, x.data_ptr(), 15, x.data_ptr(), 16, 1, x.data_ptr(), 16, None)
    assert st == api.ERR_ARG
