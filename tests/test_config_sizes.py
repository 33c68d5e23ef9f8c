"""Parity at the workload sizes the benchmark times, where the CPU oracle
cannot finish in a test: bit-exact against LELA's own results (committed
digests, tests/golden/fl_large.json) where LELA finishes in minutes, and
exact or randomised certificates at full size.

* Z/p gemm at 4096^3 and 8192^3 and the 8192 x 4096 trsm at p = 2^31 - 1
  (four limbs), by Freivalds projections (exact arithmetic);
* GF(2) gemm 16384^3 by Freivalds projections, and the echelon form of a
  32768 x 32768 matrix of planted rank 30000 by the row-space certificate;
* FaugereLachartre at m = 4000 (all four modes) and m = 8000 (reduced)
  against LELA's own outputs, and at m = 20000 by the reduced-echelon
  certificate plus agreement with the dense reduced echelon form of the
  same matrix (the reduced row-echelon form is unique, and the dense path
  shares no step with FL's split, Schur complement and back-substitution).
The counterpart of tests/test-faugere-lachartre.C:217-242 (FL output equal
to the reduced echelon form, ranks agree) at config sizes."""
import json
import os

import numpy as np
import pytest

import props
from lela_b200 import gen

HERE = os.path.dirname(os.path.abspath(__file__))


# ------------------------------------------------------------------ Z/p
@pytest.mark.gpu
@pytest.mark.parametrize("n", [4096, 8192])
def test_gemm_p31_config_size(cuda, n):
    """C <- A*B + C at p = 2147483647, M = N = K = n, the four-limb
    tensor-core kernel (16 limb products), through the host-pointer API."""
    p = 2147483647
    A = gen.dense_zp(41 + n, n, n, p)
    B = gen.dense_zp(42 + n, n, n, p)
    C = gen.dense_zp(43 + n, n, n, p)
    got = cuda.gemm(p, 1, A, B, 1, C.copy())
    assert props.freivalds_gemm(p, A, B, C, got, 1, 1)


@pytest.mark.gpu
@pytest.mark.parametrize("p", [65521, 2147483647])
def test_trsm_8192_config_size(cuda, p):
    """The trsm workload at both moduli (8192 x 8192 unit-lower L with
    uniform off-diagonal entries, 8192 x 4096 right-hand side): L X == B."""
    m, n = 8192, 4096
    L = gen.unit_lower_zp(51, m, p)
    B = gen.dense_zp(52, m, n, p)
    X = cuda.trsm(p, 1, L, B.copy(), 0, 1)
    assert props.freivalds_gemm(p, L, X, np.zeros_like(B), B, 1, 0)


# ---------------------------------------------------------------- GF(2)
@pytest.mark.gpu
def test_gf2_gemm_16384(cuda):
    """The GF(2) gemm workload, 16384^3 with Bernoulli(1/2) bits, on the
    tensor-core kernel (the default), checked by Freivalds projections."""
    n = 16384
    A = gen.dense_gf2(61, n, n)
    B = gen.dense_gf2(62, n, n)
    C = cuda.gemm_gf2(A, B, np.zeros((n, n // 64), dtype=np.uint64), n, n, 1, 0)
    assert props.freivalds_gf2(A, B, C, n, trials=3)


@pytest.mark.gpu
def test_gf2_echelon_32768_planted_rank(cuda):
    """The GF(2) echelon workload: 32768 x 32768 of planted rank 30000 (the
    product of random 32768 x 30000 and 30000 x 32768 factors, formed on the
    device).  Rank 30000, echelon structure, and the row space of the input
    inside that of the output (equal, with the rank)."""
    import torch
    m, r = 32768, 30000
    mw, rw = m // 64, (r + 63) // 64
    g = torch.Generator(device="cuda")
    g.manual_seed(71)
    rnd = lambda rows, cols: torch.randint(-2 ** 63, 2 ** 63 - 1, (rows, cols), dtype=torch.int64,
                                           device="cuda", generator=g)
    F1 = rnd(m, rw)
    F1[:, -1] &= (1 << (r % 64)) - 1
    F2 = rnd(r, mw)
    D = torch.zeros((m, mw), dtype=torch.int64, device="cuda")
    cuda.gemm_gf2(F1, F2, D, m, r, 1, 0)
    del F1, F2
    torch.cuda.synchronize()
    Dh = D.cpu().numpy().view(np.uint64).copy()
    _, rank = cuda.echelonize_gf2(D, m)
    torch.cuda.synchronize()
    assert rank == r
    E = D.cpu().numpy().view(np.uint64)
    err = props.gf2_echelon_certificate(Dh, E, rank)
    assert err is None, err


# ------------------------------------------------------ Faugere-Lachartre
def _fl_large():
    with open(os.path.join(HERE, "golden", "fl_large.json")) as f:
        return json.load(f)["cases"]


def _input_sha(X):
    import hashlib
    h = hashlib.sha256()
    for a in (X.rowptr, X.colidx, X.vals):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def _device_csr(X):
    import types
    import torch
    return types.SimpleNamespace(m=X.m, n=X.n,
                                 rowptr=torch.from_numpy(X.rowptr.view(np.int64)).cuda(),
                                 colidx=torch.from_numpy(X.colidx.view(np.int32)).cuda(),
                                 vals=torch.from_numpy(X.vals.view(np.int32)).cuda())


@pytest.mark.gpu
@pytest.mark.parametrize("case", range(5))
def test_fl_against_lela_digests(cuda, case):
    """FL at m = 4000 in all four modes and m = 8000 reduced, bit-exact in R,
    rank and det against LELA's FaugereLachartre (digests computed by
    tests/golden/make_fl_large.py from oracle/_ref)."""
    import golden_io
    import torch
    c = _fl_large()[case]
    X = gen.f4_matrix(c["seed"], c["m"], c["p"], density=c["density"])
    assert _input_sha(X) == c["input_sha"], "the generator no longer gives LELA's input"
    R, rank, det = cuda.fl_echelonize(c["p"], _device_csr(X), bool(c["reduced"]), bool(c["only_D"]))
    torch.cuda.synchronize()
    assert (rank, det) == (c["rank"], c["det"])
    got = np.ascontiguousarray(R.cpu().numpy().view(np.uint32))
    assert golden_io.sha(got) == c["R_sha"]


@pytest.mark.gpu
def test_fl_m20000_certificate(cuda):
    """The benchmark's first FL matrix (m = 20000, n = 24000, density 2.5 %):
    the reduced-echelon certificate, and equality with the dense reduced
    echelon form (unit pivots) of the same matrix computed on the GPU by the
    panel pipeline."""
    import torch
    p, m = 65521, 20000
    X = gen.f4_matrix(1000, m, p, density=0.025)
    R, rank, _ = cuda.fl_echelonize(p, _device_csr(X), True, False)
    torch.cuda.synchronize()
    err = props.rref_certificate(torch, p, X, R, rank)
    assert err is None, err
    D = torch.from_numpy(X.to_dense().view(np.int32)).cuda()
    _, drank, _ = cuda.echelonize(p, D, reduced=True, unit_pivots=True)
    torch.cuda.synchronize()
    assert drank == rank
    assert torch.equal(D, R)


@pytest.mark.gpu
def test_fl_csr_output_m20000(cuda):
    """The CSR output path at the benchmark's size, on a matrix generated on
    the device (gen.f4_matrix_torch): the CSR certificate, and equality with
    the dense output of the same matrix (expanded on the device)."""
    import torch
    from lela_b200 import certify
    p, m = 65521, 20000
    X = gen.f4_matrix_torch(77, m, p, "cuda", density=0.025)
    Rc, rank, det = cuda.fl_echelonize_csr(p, X, True, False)
    torch.cuda.synchronize()
    err = certify.rref_certificate_csr(torch, p, X, Rc, rank)
    assert err is None, err
    Rd, rank2, det2 = cuda.fl_echelonize(p, X, True, False)
    torch.cuda.synchronize()
    assert (rank2, det2) == (rank, det)
    rp = Rc.rowptr.to(torch.int64)
    rows = torch.repeat_interleave(torch.arange(Rc.m, device="cuda"), rp[1:] - rp[:-1])
    E = torch.zeros((Rd.shape[0], X.n), dtype=torch.int32, device="cuda")
    E[rows, Rc.colidx.to(torch.int64)] = Rc.vals
    assert torch.equal(E, Rd)
