"""Batched entry points: many dense echelon blocks per call (one persistent
shared-memory launch captured in a CUDA graph, plus the panel pipeline) and
many Faugere-Lachartre matrices over worker streams; every instance
bit-exact against the oracle."""
import types

import numpy as np
import pytest

import oracle
from lela_b200 import gen


def _dev(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x).view(np.int32)).cuda()


@pytest.mark.gpu
def test_echelon_batch_mixed(cuda):
    rng = np.random.default_rng(0)
    blocks, ps, kernels, wants = [], [], [], []
    for i in range(40):
        m = int(2 ** rng.uniform(3, 9))
        n = int(2 ** rng.uniform(3, 9))
        p = int(rng.choice([2, 251, 65521, 2147483647]))
        A = gen.dense_zp(i, m, n, p)
        if i % 3 == 0 and m > 4:
            A[m // 2:] = A[: m - m // 2]          # dependent rows
        if i % 5 == 0:
            A[:, : min(3, n)] = 0                  # zero leading columns
        k = [0, 0, 1, 2, 3][i % 5]
        if k == 1 and m * n * 4 > 200 * 1024:
            k = 0
        blocks.append(_dev(A)); ps.append(p); kernels.append(k)
        wants.append(oracle.echelon_zp(p, A))
    ranks, dets, st = cuda.echelonize_batch(blocks, ps, kernels)
    for i, (E, r, d) in enumerate(wants):
        assert st[i] == 0
        assert (ranks[i], dets[i]) == (r, d), i
        assert np.array_equal(blocks[i].cpu().numpy().view(np.uint32), E), i


@pytest.mark.gpu
def test_fl_batch(cuda):
    import torch
    p = 65521
    Xs, Rs, wants = [], [], []
    for i, m in enumerate([300, 800, 150, 1200, 500, 64]):
        X = gen.f4_matrix(70 + i, m, p)
        wants.append(oracle.fl_echelonize_zp(p, X.m, X.n, X.rowptr, X.colidx, X.vals, 1, 0))
        Xs.append(types.SimpleNamespace(m=X.m, n=X.n,
                                        rowptr=torch.from_numpy(X.rowptr.view(np.int64)).cuda(),
                                        colidx=_dev(X.colidx), vals=_dev(X.vals)))
        Rs.append(torch.empty((X.m, X.n), dtype=torch.int32, device="cuda"))
    ranks, dets, st = cuda.fl_echelonize_batch(Xs, [p] * len(Xs), Rs, True, nworkers=3)
    torch.cuda.synchronize()
    for i, w in enumerate(wants):
        assert st[i] == 0
        assert (ranks[i], dets[i]) == (w["rank"], w["det"]), i
        assert np.array_equal(Rs[i].cpu().numpy().view(np.uint32), w["R"]), i


@pytest.mark.gpu
def test_echelon_batch_small_kernel_edges(cuda):
    """The shared-memory kernel on tall blocks whose pivots lie more than 512
    rows down (the search covers 512 rows per pass), and on composite moduli
    where a pivot has no inverse (the reference's error, status != 0)."""
    blocks, ps, wants = [], [], []
    for i, (m, n, p) in enumerate([(1500, 20, 7), (900, 40, 65521), (700, 30, 2147483647),
                                   (60, 50, 10), (40, 40, 12), (33, 17, 9)]):
        A = gen.dense_zp(70 + i, m, n, p)
        if m > 512:
            A[: m - 100, :5] = 0               # the first columns' pivots far down
        blocks.append(_dev(A)); ps.append(p)
        try:
            wants.append(oracle.echelon_zp(p, A))
        except ArithmeticError:
            wants.append(None)
    ranks, dets, st = cuda.echelonize_batch(blocks, ps, [1] * len(blocks))
    for i, want in enumerate(wants):
        if want is None:
            assert st[i] != 0, i
            continue
        E, r, d = want
        assert st[i] == 0, i
        assert (ranks[i], dets[i]) == (r, d), i
        assert np.array_equal(blocks[i].cpu().numpy().view(np.uint32), E), i


@pytest.mark.gpu
def test_fl_batch_memory_budget(cuda):
    """The memory-budgeted queue: with a budget smaller than any matrix the
    workers run one matrix at a time and free their buffers after each; the
    results are those of the unbudgeted batch and of the oracle."""
    import torch
    p = 65521
    Xs, Rs, wants = [], [], []
    for i, m in enumerate([400, 900, 200, 650]):
        X = gen.f4_matrix(170 + i, m, p)
        wants.append(oracle.fl_echelonize_zp(p, X.m, X.n, X.rowptr, X.colidx, X.vals, 1, 0))
        Xs.append(types.SimpleNamespace(m=X.m, n=X.n,
                                        rowptr=torch.from_numpy(X.rowptr.view(np.int64)).cuda(),
                                        colidx=_dev(X.colidx), vals=_dev(X.vals)))
        Rs.append(torch.empty((X.m, X.n), dtype=torch.int32, device="cuda"))
    cuda.set_batch_memory_budget(1)
    try:
        ranks, dets, st = cuda.fl_echelonize_batch(Xs, [p] * len(Xs), Rs, True, nworkers=3)
    finally:
        cuda.set_batch_memory_budget(0)
    torch.cuda.synchronize()
    for i, w in enumerate(wants):
        assert st[i] == 0
        assert (ranks[i], dets[i]) == (w["rank"], w["det"]), i
        assert np.array_equal(Rs[i].cpu().numpy().view(np.uint32), w["R"]), i
    # the same batch again under the automatic budget
    for R in Rs:
        R.zero_()
    ranks, dets, st = cuda.fl_echelonize_batch(Xs, [p] * len(Xs), Rs, True, nworkers=3)
    torch.cuda.synchronize()
    for i, w in enumerate(wants):
        assert st[i] == 0 and (ranks[i], dets[i]) == (w["rank"], w["det"]), i
        assert np.array_equal(Rs[i].cpu().numpy().view(np.uint32), w["R"]), i
