"""Size-independent checks used where the CPU oracle cannot finish at full
size.  Each is exact; randomised ones state their error probability."""
import numpy as np


def matvec_mod(M, x, p):
    """(M @ x) mod p exactly, for entries of M and x in [0, p), p < 2^32 and
    at most 2^15 columns: x is split into 16-bit halves, so every partial
    product is below 2^48 and every row sum below 2^63 (int64)."""
    M = np.asarray(M)
    if M.dtype != np.int64:
        M = M.astype(np.int64)
    x = np.asarray(x, dtype=np.int64)
    assert M.shape[1] <= 1 << 15
    lo = (M @ (x & 0xFFFF)) % p
    hi = (M @ (x >> 16)) % p
    return (hi * 65536 + lo) % p


def freivalds_gemm(p, A, B, C0, C, a, b, trials=2, seed=0):
    """C == a*A*B + b*C0 (mod p) via random projections x: C x = a A (B x) +
    b C0 x, exact for every p < 2^32.  A wrong C passes with probability at
    most p^-trials."""
    rng = np.random.default_rng(seed)
    A = A.astype(np.int64); B = B.astype(np.int64); C0 = C0.astype(np.int64)
    C = C.astype(np.int64)
    for _ in range(trials):
        x = rng.integers(0, p, size=B.shape[1]).astype(np.int64)
        bx = matvec_mod(B, x, p)
        lhs = matvec_mod(C, x, p)
        rhs = (a * matvec_mod(A, bx, p) + b * matvec_mod(C0, x, p)) % p
        if not np.array_equal(lhs, rhs):
            return False
    return True


# ----------------------------------------------------------------- GF(2)
def gf2_matvec(M, x_words):
    """y = M x over GF(2): M packed (rows x words), x packed (words,); bit i
    of y is the parity of row i AND x."""
    return (np.bitwise_count(np.bitwise_and(M, x_words[None, :])).sum(axis=1) & 1).astype(np.uint8)


def gf2_pack_vec(bits):
    n = len(bits)
    w = (n + 63) // 64
    b = np.zeros(w * 64, dtype=np.uint8)
    b[:n] = bits
    return np.packbits(b.reshape(w, 64), axis=1, bitorder="little").view(np.uint64).reshape(w)


def freivalds_gf2(A, B, C, n, trials=2, seed=0):
    """C == A*B over GF(2) (packed words, n = columns of B and C) via random
    projections: C x = A (B x).  A wrong C passes with probability at most
    2^-trials."""
    rng = np.random.default_rng(seed)
    for _ in range(trials):
        x = rng.integers(0, 2, size=n).astype(np.uint8)
        xw = gf2_pack_vec(x)
        bx = gf2_matvec(B, xw)
        lhs = gf2_matvec(C, xw)
        rhs = gf2_matvec(A, gf2_pack_vec(bx))
        if not np.array_equal(lhs, rhs):
            return False
    return True


def gf2_row_heads(E):
    """First set bit of every row of a packed GF(2) matrix (-1: zero row)."""
    nz = E != 0
    any_nz = nz.any(axis=1)
    wi = np.argmax(nz, axis=1)
    w = E[np.arange(E.shape[0]), wi]
    low = np.bitwise_count((w & (~w + np.uint64(1))) - np.uint64(1)).astype(np.int64)
    return np.where(any_nz, wi.astype(np.int64) * 64 + low, -1)


def gf2_echelon_certificate(D, E, rank, trials=2, seed=0):
    """E (packed) is a row-echelon form of D with the given rank: rows
    0..rank-1 have strictly increasing leading columns and the rest are
    zero, and the row space of D lies in that of E (for random w, w^T D
    reduces to zero against E's rows; a D row outside E's row space passes
    with probability at most 2^-trials).  With rank = rank(D) the two row
    spaces are equal.  Returns an error string or None."""
    heads = gf2_row_heads(E)
    if (heads[rank:] != -1).any():
        return "nonzero rows below the rank"
    h = heads[:rank]
    if (h < 0).any() or (rank > 1 and not (np.diff(h) > 0).all()):
        return "leading columns not strictly increasing"
    rng = np.random.default_rng(seed)
    hw, hb = h // 64, (h % 64).astype(np.uint64)
    for t in range(trials):
        sel = rng.integers(0, 2, size=D.shape[0]).astype(bool)
        v = np.bitwise_xor.reduce(D[sel], axis=0) if sel.any() else np.zeros(D.shape[1], np.uint64)
        v = v.copy()
        for i in range(rank):
            if (v[hw[i]] >> hb[i]) & np.uint64(1):
                v ^= E[i]
        if v.any():
            return "a combination of D's rows is not in E's row space (trial %d)" % t
    return None


# ---------------------------------------------------------- Z/p, reduced
from lela_b200.certify import csr_vecmat_mod, rref_certificate  # noqa: E402,F401
