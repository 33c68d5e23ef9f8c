"""lela_cuda_gemm_zp_u32_noalloc: the Z/p tensor-core gemm for callers that
cannot allocate device memory (their device memory belongs to a host
framework's allocator or a fixed budget, or cudaMalloc's possible device
synchronisation is not allowed on their path).  The entry point keeps its
scratch in a fixed array inside the library; this test calls it through the
C ABI twice in a row and compares each result with the regular device-pointer
entry point lela_cuda_gemm_zp_u32_dev (bit-exact, as every Z/p test here).

The file name sorts last so that a run stopping at the first failure has
already run every other test; it also passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from lela_b200 import api, gen

_P = ctypes.c_void_p
_S = ctypes.c_size_t
_U = ctypes.c_uint32


def _noalloc_fn():
    fn = api.load_library().lela_cuda_gemm_zp_u32_noalloc
    fn.argtypes = [_S, _S, _S, _U, _U, _P, _S, _P, _S, _U, _P, _S, _P]
    fn.restype = ctypes.c_int
    return fn


@pytest.mark.gpu
def test_noalloc_matches_dev_entry_point_twice():
    import torch
    fn = _noalloc_fn()
    cm = api.CudaModule(0)
    dev = torch.device("cuda", 0)
    t = lambda x: torch.from_numpy(x.view(np.int32)).to(dev)
    cases = [(65521, 700, 650, 900, 3, 5), (2147483647, 300, 257, 1000, 1, 1)]
    try:
        for i, (p, m, n, k, a, b) in enumerate(cases):
            A = gen.dense_zp(500 + i, m, k, p)
            B = gen.dense_zp(600 + i, k, n, p)
            C = gen.dense_zp(700 + i, m, n, p)
            dA, dB = t(A), t(B)
            ref_C, new_C = t(C), t(C)
            cm.gemm(p, a, dA, dB, b, ref_C)
            cm.synchronize()
            torch.cuda.synchronize()
            st = fn(m, n, k, p, a, dA.data_ptr(), k, dB.data_ptr(), n, b, new_C.data_ptr(), n, None)
            assert st == api.OK, st
            torch.cuda.synchronize()
            assert torch.equal(ref_C, new_C), "call %d differs from lela_cuda_gemm_zp_u32_dev" % i
    finally:
        cm.close()


@pytest.mark.gpu
def test_noalloc_rejects_sizes_beyond_scratch():
    import torch
    fn = _noalloc_fn()
    x = torch.zeros(16, dtype=torch.int32, device="cuda")
    # 2 limbs * (20000 + 20000) rows * 4096 bytes > 64 MiB
    st = fn(20000, 20000, 4096, 65521, 1, x.data_ptr(), 4096, x.data_ptr(), 20000, 1,
            x.data_ptr(), 20000, None)
    assert st == api.ERR_ARG
