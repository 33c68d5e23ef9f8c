"""Randomised certificates for results of the exact path at sizes where no
CPU implementation can recompute them in reasonable time.

rref_certificate checks that a device matrix R is the reduced row-echelon
form of a sparse matrix X over Z/p: the echelon structure exactly, and the
row-space inclusion by random projections (the test of
tests/test-faugere-lachartre.C:217-242, FL output against the reduced
echelon form, at sizes where that reference form cannot be computed on a
CPU).  The check runs on numpy (the CSR side) and on the device in float64
(exact below 2^53); it does not use this library's kernels.
"""
import numpy as np


def csr_vecmat_mod(X, w, p):
    """w^T X mod p for a CSR matrix X over Z/p (w of length X.m, entries in
    [0, p), p < 2^16): the products are below 2^32 and the column sums below
    2^53, so float64 accumulation is exact."""
    rows = np.repeat(np.arange(X.m), np.diff(X.rowptr).astype(np.int64))
    prod = (w[rows].astype(np.int64) * X.vals.astype(np.int64)) % p
    v = np.bincount(X.colidx.astype(np.int64), weights=prod.astype(np.float64), minlength=X.n)
    return (v.astype(np.int64) % p)


def rref_certificate(torch, p, X, R, rank, trials=2, seed=0):
    """R (a torch CUDA tensor, int32 storage, X.m x X.n) is the reduced
    row-echelon form of the CSR matrix X over Z/p (p < 2^16) with the given
    rank: (1) rows 0..rank-1 have strictly increasing leading columns holding
    1 and every other entry of those pivot columns is 0, rows from rank on
    are zero; (2) X's row space lies in R's: for random w, w^T X minus its
    combination of R's rows by the pivot-column entries is zero (a row of X
    outside R's row space passes with probability at most p^-trials).  The
    inclusion the other way needs rank(R) = rank(X); the tests add it by
    comparing with an independent computation.  Returns an error string or
    None."""
    m, n = R.shape
    nz = R != 0
    rows_nz = nz.any(dim=1)
    if int(rows_nz.sum()) != rank or (rank and not bool(rows_nz[:rank].all())):
        return "nonzero rows do not match the rank"
    if rank == 0:
        return None
    heads = nz[:rank].to(torch.uint8).argmax(dim=1)
    if rank > 1 and not bool((heads[1:] > heads[:-1]).all()):
        return "leading columns not strictly increasing"
    lead = R[torch.arange(rank, device=R.device), heads]
    if not bool((lead == 1).all()):
        return "a leading entry is not 1"
    if not bool((nz[:, heads].sum(dim=0) == 1).all()):
        return "a pivot column has another nonzero"
    rng = np.random.default_rng(seed)
    hcpu = heads.cpu().numpy()
    for t in range(trials):
        w = rng.integers(0, p, size=X.m)
        v = csr_vecmat_mod(X, w, p)
        coef = torch.from_numpy(v[hcpu].astype(np.float64)).to(R.device)
        # v - coef^T R, in float64 (exact: sums below 2^53), row chunks of R
        acc = torch.zeros(n, dtype=torch.float64, device=R.device)
        step = 4096
        for r0 in range(0, rank, step):
            r1 = min(rank, r0 + step)
            blk = R[r0:r1].to(torch.int64).to(torch.float64)
            acc += coef[r0:r1] @ blk
        red = (torch.from_numpy(v.astype(np.float64)).to(R.device) - torch.remainder(acc, p))
        if bool((torch.remainder(red, p) != 0).any()):
            return "w^T X is not in R's row space (trial %d)" % t
    return None


def rref_certificate_csr(torch, p, X, R, rank, trials=2, seed=0, chunk=1 << 26):
    """rref_certificate for a result given as CSR rows on the device (R with
    m, n and tensors rowptr (int64), colidx, vals (int32 storage), as
    CudaModule.fl_echelonize_csr returns it) and X as device CSR tensors of
    the same form: (1) rows 0..rank-1 are nonempty, their first entries lie
    in strictly increasing columns and are 1, each such pivot column holds
    no other entry, rows from rank on are empty; (2) for random w, w^T X
    minus its combination of R's rows by the pivot-column entries is zero
    (float64 sums on the device, exact below 2^53: p < 2^16 and fewer than
    2^21 rows).  Entries are processed about `chunk` at a time, so results
    with billions of entries fit beside the matrices.  Returns an error
    string or None."""
    dev = R.rowptr.device
    rp = R.rowptr.to(torch.int64)
    lens = rp[1:] - rp[:-1]
    if int((lens > 0).sum()) != rank or (rank and not bool((lens[:rank] > 0).all())):
        return "nonempty rows do not match the rank"
    if rank == 0:
        return None
    heads = R.colidx[rp[:rank]].to(torch.int64)
    if rank > 1 and not bool((heads[1:] > heads[:-1]).all()):
        return "leading columns not strictly increasing"
    if not bool((R.vals[rp[:rank]] == 1).all()):
        return "a leading entry is not 1"
    is_pc = torch.zeros(R.n, dtype=torch.bool, device=dev)
    is_pc[heads] = True

    def row_chunks(rowptr, m):
        """(r0, r1, e0, e1): consecutive rows holding about `chunk` entries."""
        r0 = 0
        while r0 < m:
            e0 = int(rowptr[r0])
            r1 = int(torch.searchsorted(rowptr, torch.tensor(e0 + chunk, device=dev), right=True)) - 1
            r1 = min(m, max(r1, r0 + 1))
            yield r0, r1, e0, int(rowptr[r1])
            r0 = r1

    pc_entries = 0
    for r0, r1, e0, e1 in row_chunks(rp, R.m):
        pc_entries += int(is_pc[R.colidx[e0:e1].to(torch.int64)].sum())
    if pc_entries != rank:
        return "a pivot column has another nonzero"
    xrp = X.rowptr.to(torch.int64)
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    for t in range(trials):
        w = torch.randint(0, p, (X.m,), generator=g, device=dev, dtype=torch.int64)
        v = torch.zeros(X.n, dtype=torch.float64, device=dev)
        for r0, r1, e0, e1 in row_chunks(xrp, X.m):
            rows = torch.repeat_interleave(torch.arange(r0, r1, device=dev), xrp[r0 + 1:r1 + 1] - xrp[r0:r1])
            prod = (w[rows] * X.vals[e0:e1].to(torch.int64)) % p
            v.index_add_(0, X.colidx[e0:e1].to(torch.int64), prod.to(torch.float64))
        v = torch.remainder(v, p)
        coef = v[heads]                         # per pivot row
        acc = torch.zeros(R.n, dtype=torch.float64, device=dev)
        for r0, r1, e0, e1 in row_chunks(rp, min(R.m, rank)):
            rows = torch.repeat_interleave(torch.arange(r0, r1, device=dev), rp[r0 + 1:r1 + 1] - rp[r0:r1])
            acc.index_add_(0, R.colidx[e0:e1].to(torch.int64),
                           coef[rows] * R.vals[e0:e1].to(torch.float64))
        if bool((torch.remainder(v - torch.remainder(acc, p), p) != 0).any()):
            return "w^T X is not in R's row space (trial %d)" % t
    return None
