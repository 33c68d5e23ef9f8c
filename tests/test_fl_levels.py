"""The dependency structure of Faugere-Lachartre's pivot block A on the
bench's F4 matrices (lela_b200.gen.f4_matrix, m = 20000, density 2.5 %).

FL solves A^-1 B with A the upper-triangular pivot block (faugere-
lachartre.tcc:791, level3-generic.tcc:421-498).  A level-set (row-by-row)
sparse solve can process at once only the rows whose dependencies are all
solved: row i of the back substitution waits for every pivot j > i at one
of its off-diagonal pivot columns, so the number of dependent steps is the
longest such chain.  This test measures that chain on the first matrix the
FL bench line times, which is what rules the level-set form out here: about
7500 levels of at most about ten rows each, so even one microsecond per
level (a grid-wide barrier) costs more than the whole tiled tensor-core
solve of the same block.  CPU only."""
import numpy as np

from lela_b200 import gen


def pivot_block_levels(X):
    """(pivots, off-diagonal nonzeros of A, level of each pivot row) for the
    back substitution with FL's pivot block: pivot rows are the rows whose
    head is larger than the previous row's (setup_splicer, faugere-
    lachartre.tcc:47-146), A's columns the pivot columns."""
    rp = X.rowptr.astype(np.int64)
    ci = X.colidx.astype(np.int64)
    heads = ci[rp[:-1]]
    piv = np.concatenate([[True], heads[1:] > heads[:-1]])
    prow = np.flatnonzero(piv)
    index = -np.ones(X.n, np.int64)
    index[heads[prow]] = np.arange(len(prow))
    level = np.zeros(len(prow), np.int64)
    nnz = 0
    for i in range(len(prow) - 1, -1, -1):
        r = prow[i]
        js = index[ci[rp[r] + 1: rp[r + 1]]]
        js = js[js >= 0]
        nnz += len(js)
        if len(js):
            level[i] = 1 + level[js].max()
    return len(prow), nnz, level


def test_fl_pivot_block_is_a_long_chain():
    X = gen.f4_matrix(1000, 20000, 65521, density=0.025)
    npiv, nnz, level = pivot_block_levels(X)
    counts = np.bincount(level)
    assert npiv == 15000
    assert nnz > 5_000_000
    assert len(counts) > 7000            # dependent steps of a level-set solve
    assert counts.max() <= 16            # rows solvable together in one step
    assert np.median(counts) <= 3


def test_levels_of_a_small_chain():
    """The level computation on a hand-made 4-pivot staircase: row 0
    depends on 1 and 3, row 1 on 2, row 2 on nothing, row 3 on nothing;
    plus a non-pivot row (same head as row 1) that A does not contain."""
    rows = [[0, 1, 3], [1, 2], [1, 4], [2, 5], [3]]
    rowptr = np.zeros(len(rows) + 1, np.uint64)
    rowptr[1:] = np.cumsum([len(r) for r in rows])
    colidx = np.concatenate([np.array(r, np.uint32) for r in rows])
    X = gen.CSR(len(rows), 6, rowptr, colidx, np.ones(len(colidx), np.uint32))
    npiv, nnz, level = pivot_block_levels(X)
    assert npiv == 4 and nnz == 3
    assert level.tolist() == [2, 1, 0, 0]
