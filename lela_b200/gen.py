"""Seeded synthetic inputs for the exact linear-algebra hot path.

Every generator is a pure function of its arguments (numpy PCG64 streams),
so the CUDA path, the CPU oracle and LELA's own code see identical inputs.
Shapes and value distributions follow the workloads the reference's path is
exercised on: dense Z/p matrices with i.i.d. uniform entries in [0, p),
triangular systems, GF(2) Bernoulli(1/2) bit matrices packed LittleEndian
(bit j of 64-bit word w is column 64w+j, as LELA's BitVector<LittleEndian>
stores it), and F4-shaped sparse matrices in the row-sorted staircase form
that FaugereLachartre::echelonize requires (lela/algorithms/
faugere-lachartre.tcc:61-117).
"""
import numpy as np


def rng(seed):
    return np.random.Generator(np.random.PCG64(seed))


def dense_zp(seed, m, n, p):
    """m x n uint32 matrix, entries i.i.d. uniform in [0, p)."""
    return rng(seed).integers(0, p, size=(m, n), dtype=np.uint32)


def unit_lower_zp(seed, m, p):
    """m x m unit-lower-triangular matrix, off-diagonal uniform in [0, p)."""
    L = np.tril(dense_zp(seed, m, m, p), -1)
    np.fill_diagonal(L, 1)
    return L


def upper_zp(seed, m, p, unit=False):
    """m x m upper-triangular matrix with nonzero diagonal (or unit)."""
    g = rng(seed)
    U = np.triu(g.integers(0, p, size=(m, m), dtype=np.uint32), 1)
    d = np.ones(m, dtype=np.uint32) if unit else g.integers(1, p, size=m, dtype=np.uint32)
    U[np.arange(m), np.arange(m)] = d
    return U


def words(n):
    return (n + 63) // 64


def dense_gf2(seed, m, n):
    """m x n GF(2) matrix of Bernoulli(1/2) bits, packed into uint64 words."""
    W = rng(seed).integers(0, 2**63, size=(m, words(n)), dtype=np.uint64, endpoint=True)
    W = W | (rng(seed + 1).integers(0, 2, size=(m, words(n)), dtype=np.uint64) << np.uint64(63))
    if n & 63:
        W[:, -1] &= np.uint64((1 << (n & 63)) - 1)
    return W


def pack_gf2(bits):
    """Pack a 0/1 array (m x n) into LittleEndian uint64 words."""
    bits = np.asarray(bits, dtype=np.uint8)
    m, n = bits.shape
    w = words(n)
    padded = np.zeros((m, w * 64), dtype=np.uint8)
    padded[:, :n] = bits
    b = np.packbits(padded.reshape(m, w, 64), axis=2, bitorder="little")
    return b.view(np.uint64).reshape(m, w)


def unpack_gf2(W, n):
    W = np.ascontiguousarray(W, dtype=np.uint64)
    m = W.shape[0]
    b = np.unpackbits(W.view(np.uint8).reshape(m, -1), axis=1, bitorder="little")
    return b[:, :n]


def planted_rank_gf2(seed, m, n, r):
    """m x n GF(2) matrix of rank r (w.h.p.): product of random m x r and
    r x n factors, computed with packed word arithmetic."""
    g = rng(seed)
    F1 = g.integers(0, 2, size=(m, r), dtype=np.uint8)
    F2 = pack_gf2(g.integers(0, 2, size=(r, n), dtype=np.uint8))
    out = np.zeros((m, words(n)), dtype=np.uint64)
    for i in range(m):
        sel = np.nonzero(F1[i])[0]
        if len(sel):
            out[i] = np.bitwise_xor.reduce(F2[sel], axis=0)
    return out


class CSR:
    """Row-sorted CSR matrix over Z/p: rowptr (m+1, uint64), colidx (uint32),
    vals (uint32).  Column indices within a row are strictly increasing."""

    def __init__(self, m, n, rowptr, colidx, vals):
        self.m, self.n = int(m), int(n)
        self.rowptr = np.ascontiguousarray(rowptr, dtype=np.uint64)
        self.colidx = np.ascontiguousarray(colidx, dtype=np.uint32)
        self.vals = np.ascontiguousarray(vals, dtype=np.uint32)

    @property
    def nnz(self):
        return int(self.rowptr[-1])

    def to_dense(self):
        D = np.zeros((self.m, self.n), dtype=np.uint32)
        rows = np.repeat(np.arange(self.m), np.diff(self.rowptr).astype(np.int64))
        D[rows, self.colidx.astype(np.int64)] = self.vals
        return D

    @staticmethod
    def from_dense(D):
        D = np.asarray(D, dtype=np.uint32)
        m, n = D.shape
        nz = D != 0
        rowptr = np.zeros(m + 1, dtype=np.uint64)
        rowptr[1:] = np.cumsum(nz.sum(axis=1))
        r, c = np.nonzero(nz)
        return CSR(m, n, rowptr, c.astype(np.uint32), D[r, c])


def f4_matrix(seed, m, p, n=None, density=None, pivot_frac=0.75, dep_frac=0.05):
    """F4-shaped sparse matrix over Z/p in FaugereLachartre input form.

    * n = floor(1.2 m) columns unless given;
    * round(pivot_frac * m) pivot rows whose leading columns are distinct,
      chosen uniformly without replacement and sorted, leading value 1;
    * every other row copies the leading column of a uniformly chosen pivot
      row and is placed directly after it (leading value uniform in [1, p));
    * each row holds ~density * n further nonzeros right of its leading
      column, clustered towards it (exponential offsets), values uniform in
      [1, p); density is drawn per matrix from [1%, 4%] unless given;
    * dep_frac of the non-pivot rows are replaced by c1 * (pivot row with the
      same leading column) + c2 * (a later pivot row), which makes them
      linearly dependent (rank deficiency of the Schur complement).
    """
    g = rng(seed)
    n = int(1.2 * m) if n is None else int(n)
    if density is None:
        density = float(g.uniform(0.01, 0.04))
    npiv = int(round(pivot_frac * m))
    npiv = max(0, min(npiv, n, m))
    nnp = m - npiv
    lead = np.sort(g.choice(n, size=npiv, replace=False)) if npiv else np.zeros(0, np.int64)
    owner = np.sort(g.integers(0, npiv, size=nnp)) if (npiv and nnp) else np.zeros(0, np.int64)
    # row order: pivot row i, then the non-pivot rows that copy its head
    counts = np.bincount(owner, minlength=npiv) if npiv else np.zeros(0, np.int64)
    heads = np.repeat(lead, counts + 1) if npiv else np.zeros(0, np.int64)
    is_piv = np.zeros(len(heads), dtype=bool)
    if npiv:
        starts = np.concatenate([[0], np.cumsum(counts + 1)[:-1]])
        is_piv[starts] = True
    mm = len(heads)
    per_row = max(1, int(round(density * n)))
    rows_c, rows_v = [], []
    for i in range(mm):
        h = int(heads[i])
        room = n - h - 1
        k = min(per_row, room)
        if k > 0:
            off = np.unique((g.exponential(scale=max(1.0, room / 4.0), size=2 * k)).astype(np.int64))
            off = off[off < room][:k]
            cols = h + 1 + off
        else:
            cols = np.zeros(0, np.int64)
        v = g.integers(1, p, size=len(cols), dtype=np.uint32)
        lead_v = 1 if is_piv[i] else int(g.integers(1, p))
        rows_c.append(np.concatenate([[h], cols]).astype(np.uint32))
        rows_v.append(np.concatenate([[lead_v], v]).astype(np.uint32))
    # planted dependencies
    np_rows = np.nonzero(~is_piv)[0]
    ndep = int(round(dep_frac * len(np_rows)))
    if ndep and npiv > 1:
        piv_rows = np.nonzero(is_piv)[0]
        piv_of_head = {int(heads[r]): int(r) for r in piv_rows}
        for r in g.choice(np_rows, size=ndep, replace=False):
            h = int(heads[r])
            r1 = piv_of_head[h]
            later = piv_rows[heads[piv_rows] > h]
            if len(later) == 0:
                continue
            r2 = int(g.choice(later))
            c1 = int(g.integers(1, p)); c2 = int(g.integers(1, p))
            acc = {}
            for rr, cc in ((r1, c1), (r2, c2)):
                for col, val in zip(rows_c[rr].tolist(), rows_v[rr].tolist()):
                    acc[col] = (acc.get(col, 0) + cc * val) % p
            cols = np.array(sorted(c for c, v in acc.items() if v), dtype=np.uint32)
            rows_c[r] = cols
            rows_v[r] = np.array([acc[c] for c in cols.tolist()], dtype=np.uint32)
    lens = np.array([len(c) for c in rows_c], dtype=np.uint64)
    rowptr = np.zeros(mm + 1, dtype=np.uint64)
    rowptr[1:] = np.cumsum(lens)
    colidx = np.concatenate(rows_c) if mm else np.zeros(0, np.uint32)
    vals = np.concatenate(rows_v) if mm else np.zeros(0, np.uint32)
    return CSR(mm, n, rowptr, colidx, vals)


def f4_matrix_small(seed, m, n, p, density=0.1):
    """The staircase family of the reference's own FL test
    (tests/test-faugere-lachartre.C:142-175, restated with numpy streams):
    walking down the rows, the leading column stays (1/7), advances by one
    (5/7) or jumps forward (1/7); each row is random right of its head with
    the given density; rows stop once the head would leave the matrix."""
    g = rng(seed)
    col = 0
    rows_c, rows_v = [], []
    for i in range(m):
        v = int(g.integers(0, 7))
        if 1 <= v <= 5:
            col += 1
        elif v == 6:
            hi = n - (m - i + 1)
            if hi > col:
                col = int(g.integers(col, hi))
        if col >= n:
            rows_c.append(np.zeros(0, np.uint32)); rows_v.append(np.zeros(0, np.uint32))
            continue
        rest = np.arange(col + 1, n)
        keep = rest[g.random(len(rest)) < density]
        cols = np.concatenate([[col], keep]).astype(np.uint32)
        vals = g.integers(1, p, size=len(cols), dtype=np.uint32)
        rows_c.append(cols); rows_v.append(vals)
    lens = np.array([len(c) for c in rows_c], dtype=np.uint64)
    rowptr = np.zeros(m + 1, dtype=np.uint64)
    rowptr[1:] = np.cumsum(lens)
    return CSR(m, n, rowptr, np.concatenate(rows_c), np.concatenate(rows_v))


def f4_matrix_fast(seed, m, p, n=None, density=None, pivot_frac=0.75, dep_frac=0.05):
    """The F4 family of f4_matrix (same pivot structure, density, value
    distribution and planted dependencies), generated with whole-array
    operations so that matrices with m in the tens of thousands take well
    under a second.  The offsets right of each row's leading column are
    cumulative sums of geometric gaps (strictly increasing, clustered
    towards the leading column) instead of sorted distinct exponential
    draws, so for a given seed the matrix differs from f4_matrix's."""
    g = rng(seed)
    n = int(1.2 * m) if n is None else int(n)
    if density is None:
        density = float(g.uniform(0.01, 0.04))
    npiv = max(0, min(int(round(pivot_frac * m)), n, m))
    nnp = m - npiv
    lead = np.sort(g.choice(n, size=npiv, replace=False)) if npiv else np.zeros(0, np.int64)
    owner = np.sort(g.integers(0, npiv, size=nnp)) if (npiv and nnp) else np.zeros(0, np.int64)
    counts = np.bincount(owner, minlength=npiv) if npiv else np.zeros(0, np.int64)
    heads = np.repeat(lead, counts + 1).astype(np.int64) if npiv else np.zeros(0, np.int64)
    is_piv = np.zeros(len(heads), dtype=bool)
    if npiv:
        starts = np.concatenate([[0], np.cumsum(counts + 1)[:-1]])
        is_piv[starts] = True
    mm = len(heads)
    k = max(1, int(round(density * n)))
    room = n - heads - 1
    # gaps with mean room / (4 k): the k offsets spread over about a quarter
    # of the room, more densely near the leading column
    mean_gap = np.maximum(1.0, room / (4.0 * k))
    gaps = 1 + np.floor(g.exponential(size=(mm, k)) * (mean_gap[:, None] - 1.0 + 1e-9)).astype(np.int64)
    off = np.cumsum(gaps, axis=1) - 1
    valid = off < room[:, None]
    cols = heads[:, None] + 1 + off
    vals = g.integers(1, p, size=(mm, k), dtype=np.uint32)
    lead_v = np.where(is_piv, 1, g.integers(1, p, size=mm)).astype(np.uint32)
    lens = 1 + valid.sum(axis=1)
    rowptr = np.zeros(mm + 1, dtype=np.uint64)
    rowptr[1:] = np.cumsum(lens)
    colidx = np.empty(int(rowptr[-1]), dtype=np.uint32)
    vv = np.empty(int(rowptr[-1]), dtype=np.uint32)
    first = rowptr[:-1].astype(np.int64)
    colidx[first] = heads
    vv[first] = lead_v
    body = np.ones(int(rowptr[-1]), dtype=bool)
    body[first] = False
    colidx[body] = cols[valid]
    vv[body] = vals[valid]
    X = CSR(mm, n, rowptr, colidx, vv)
    # planted dependencies: c1 * (pivot row of the same head) + c2 * (a later
    # pivot row), as in f4_matrix
    np_rows = np.nonzero(~is_piv)[0]
    ndep = int(round(dep_frac * len(np_rows)))
    if not (ndep and npiv > 1):
        return X
    piv_rows = np.nonzero(is_piv)[0]
    piv_of = np.searchsorted(lead, heads)  # index among pivot rows of each row's head
    rows_c = {}
    for r in g.choice(np_rows, size=ndep, replace=False):
        i1 = int(piv_of[r])
        if i1 + 1 >= npiv:
            continue
        r1, r2 = int(piv_rows[i1]), int(piv_rows[int(g.integers(i1 + 1, npiv))])
        c1, c2 = int(g.integers(1, p)), int(g.integers(1, p))
        a0, a1 = int(rowptr[r1]), int(rowptr[r1 + 1])
        b0, b1 = int(rowptr[r2]), int(rowptr[r2 + 1])
        cc = np.concatenate([colidx[a0:a1], colidx[b0:b1]]).astype(np.int64)
        vals2 = np.concatenate([(vv[a0:a1].astype(np.uint64) * c1) % p,
                                (vv[b0:b1].astype(np.uint64) * c2) % p])
        u, inv = np.unique(cc, return_inverse=True)
        acc = np.zeros(len(u), dtype=np.uint64)
        np.add.at(acc, inv, vals2)
        acc %= p
        keep = acc != 0
        rows_c[int(r)] = (u[keep].astype(np.uint32), acc[keep].astype(np.uint32))
    if not rows_c:
        return X
    lens = np.diff(rowptr).astype(np.int64)
    for r, (c_, v_) in rows_c.items():
        lens[r] = len(c_)
    rp2 = np.zeros(mm + 1, dtype=np.uint64)
    rp2[1:] = np.cumsum(lens)
    ci2 = np.empty(int(rp2[-1]), dtype=np.uint32)
    v2 = np.empty(int(rp2[-1]), dtype=np.uint32)
    keep_rows = np.ones(mm, dtype=bool)
    keep_rows[list(rows_c)] = False
    src_rows = np.repeat(keep_rows, np.diff(rowptr).astype(np.int64))
    dst_rows = np.repeat(keep_rows, lens)
    ci2[dst_rows] = colidx[src_rows]
    v2[dst_rows] = vv[src_rows]
    for r, (c_, v_) in rows_c.items():
        ci2[int(rp2[r]):int(rp2[r + 1])] = c_
        v2[int(rp2[r]):int(rp2[r + 1])] = v_
    return CSR(mm, n, rp2, ci2, v2)


def f4_matrix_torch(seed, m, p, device, n=None, density=0.025, pivot_frac=0.75, dep_frac=0.05):
    """f4_matrix_fast's family generated on a torch device (for matrices
    too large for host-side generation: m = 120000 has about 4.3e8
    nonzeros).  Same structure -- staircase of pivot rows with leading 1,
    non-pivot rows copying a pivot row's leading column right after it,
    clustered nonzeros right of the leading column, values uniform in
    [1, p), dep_frac of the non-pivot rows planted as combinations of two
    pivot rows -- from torch's generator, so the matrix differs from the
    numpy generators' for the same seed.  Returns an object with m, n and
    CSR tensors rowptr (int64), colidx, vals (int32 storage) on the
    device."""
    import types
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    n = int(1.2 * m) if n is None else int(n)
    npiv = max(0, min(int(round(pivot_frac * m)), n, m))
    nnp = m - npiv
    lead = torch.sort(torch.randperm(n, generator=g, device=device)[:npiv]).values
    owner = torch.sort(torch.randint(0, npiv, (nnp,), generator=g, device=device)).values
    counts = torch.bincount(owner, minlength=npiv)
    heads = torch.repeat_interleave(lead, counts + 1)
    starts = torch.cumsum(counts + 1, 0) - (counts + 1)
    is_piv = torch.zeros(len(heads), dtype=torch.bool, device=device)
    is_piv[starts] = True
    mm = len(heads)
    k = max(1, int(round(density * n)))
    room = (n - heads - 1).to(torch.float32)
    mean_gap = torch.clamp(room / (4.0 * k), min=1.0)
    rowptr = torch.zeros(mm + 1, dtype=torch.int64, device=device)
    cols_all, vals_all, lens = [], [], torch.empty(mm, dtype=torch.int64, device=device)
    step = max(1, (1 << 26) // k)  # rows per chunk: about 6.7e7 draws at a time
    for r0 in range(0, mm, step):
        r1 = min(mm, r0 + step)
        e = torch.empty((r1 - r0, k), dtype=torch.float32, device=device).exponential_(generator=g)
        gaps = 1 + torch.floor(e * (mean_gap[r0:r1, None] - 1.0 + 1e-6)).to(torch.int64)
        off = torch.cumsum(gaps, 1) - 1
        del e, gaps
        valid = off < (n - heads[r0:r1] - 1)[:, None]
        c = heads[r0:r1, None] + 1 + off
        v = torch.randint(1, p, (r1 - r0, k), generator=g, device=device, dtype=torch.int64)
        lv = torch.where(is_piv[r0:r1], torch.ones_like(heads[r0:r1]),
                         torch.randint(1, p, (r1 - r0,), generator=g, device=device))
        # each row: its head, then its valid offsets
        c = torch.cat([heads[r0:r1, None], torch.where(valid, c, -1)], 1)
        v = torch.cat([lv[:, None], v], 1)
        keep = c >= 0
        lens[r0:r1] = keep.sum(1)
        cols_all.append(c[keep].to(torch.int32))
        vals_all.append(v[keep].to(torch.int32))
        del c, v, keep, valid, off
    rowptr[1:] = torch.cumsum(lens, 0)
    colidx = torch.cat(cols_all)
    vals = torch.cat(vals_all)
    del cols_all, vals_all
    # planted dependencies: c1 * (pivot row of the same head) + c2 * (a later pivot row)
    np_rows = torch.nonzero(~is_piv).flatten()
    ndep = int(round(dep_frac * len(np_rows)))
    if ndep and npiv > 1:
        piv_rows = torch.nonzero(is_piv).flatten()
        piv_of = torch.searchsorted(lead, heads)
        pick = np_rows[torch.randperm(len(np_rows), generator=g, device=device)[:ndep]]
        repl = {}
        for r in pick.tolist():
            i1 = int(piv_of[r])
            if i1 + 1 >= npiv:
                continue
            i2 = int(torch.randint(i1 + 1, npiv, (1,), generator=g, device=device))
            c1, c2 = (int(x) for x in torch.randint(1, p, (2,), generator=g, device=device))
            r1_, r2_ = int(piv_rows[i1]), int(piv_rows[i2])
            a0, a1 = int(rowptr[r1_]), int(rowptr[r1_ + 1])
            b0, b1 = int(rowptr[r2_]), int(rowptr[r2_ + 1])
            cc = torch.cat([colidx[a0:a1], colidx[b0:b1]]).to(torch.int64)
            vv = torch.cat([vals[a0:a1].to(torch.int64) * c1 % p, vals[b0:b1].to(torch.int64) * c2 % p])
            u, inv = torch.unique(cc, return_inverse=True)
            acc = torch.zeros(len(u), dtype=torch.int64, device=device).index_add_(0, inv, vv) % p
            nz = acc != 0
            repl[r] = (u[nz].to(torch.int32), acc[nz].to(torch.int32))
        if repl:
            new_lens = lens.clone()
            for r, (cc, _) in repl.items():
                new_lens[r] = len(cc)
            rp2 = torch.zeros(mm + 1, dtype=torch.int64, device=device)
            rp2[1:] = torch.cumsum(new_lens, 0)
            keep_row = torch.ones(mm, dtype=torch.bool, device=device)
            keep_row[torch.tensor(list(repl), device=device)] = False
            src_keep = torch.repeat_interleave(keep_row, lens)
            dst_keep = torch.repeat_interleave(keep_row, new_lens)
            ci2 = torch.empty(int(rp2[-1]), dtype=torch.int32, device=device)
            v2 = torch.empty_like(ci2)
            ci2[dst_keep] = colidx[src_keep]
            v2[dst_keep] = vals[src_keep]
            for r, (cc, vv) in repl.items():
                ci2[int(rp2[r]):int(rp2[r + 1])] = cc
                v2[int(rp2[r]):int(rp2[r + 1])] = vv
            rowptr, colidx, vals = rp2, ci2, v2
    return types.SimpleNamespace(m=mm, n=n, rowptr=rowptr, colidx=colidx, vals=vals,
                                 nnz=int(rowptr[-1]))
