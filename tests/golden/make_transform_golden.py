"""Generate tests/golden/transform_golden.npz, gj_transform_golden.npz and
packed_golden.npz from LELA's own CPU code: Elimination::echelonize_reduced
(A, L, P, rank, det, compute_L = true) (lela/algorithms/elimination.tcc:
143-265), GaussJordan::echelonize_reduced (A, L, P, rank, det) (lela/
algorithms/gauss-jordan.tcc:434-466), and the non-reduced forms that keep L
below the diagonal, Elimination::echelonize (A, P, rank, det) with its
default compute_L and GaussJordan::echelonize (A, P, rank, det), through
oracle/_ref/liblela_ref.so.

    python tests/golden/make_transform_golden.py

Inputs are seeded uniform residues (lela_b200.gen.dense_zp) shaped as the
cases the transform has: square, tall and wide, rank deficient (a product of
thin factors), zero column bands and zero rows, pivots far below the current
row, empty matrices, and LELA's pivot-inversion failures (a composite
modulus, p >= 2^31).  Each case keeps A, and LELA's R, L, P, rank, det and
status (0, or -1 when LELA throws).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from lela_b200 import gen  # noqa: E402

SHAPES = [(1, 1), (0, 5), (5, 0), (9, 9), (14, 6), (6, 14), (40, 33), (33, 70)]
MODULI = [2, 3, 251, 65521, 65536, 2147483647, 4294967291]


def case_matrix(seed, m, n, p, kind):
    A = gen.dense_zp(seed, m, n, p)
    if m == 0 or n == 0:
        return A
    if kind == 1:  # rank deficient
        r = max(1, min(m, n) // 3)
        F = gen.dense_zp(seed + 1, m, r, p).astype(object) @ gen.dense_zp(seed + 2, r, n, p).astype(object)
        A = (F % p).astype(np.uint32)
    elif kind == 2:  # zero columns and rows, pivots far below
        A[:, ::3] = 0
        A[: m // 2, : n // 2] = 0
        A[m - 1] = 0
    return A


def write(fn, fname):
    out = {}
    names = []
    for pi, p in enumerate(MODULI):
        for si, (m, n) in enumerate(SHAPES):
            for kind in range(3):
                if (m == 0 or n == 0) and kind:
                    continue
                seed = 1000 * pi + 10 * si + kind
                A = case_matrix(seed, m, n, p, kind)
                pre = "tl%d_%d_%d_" % (pi, si, kind)
                try:
                    R, L, P, r, d = fn(p, A)
                    st = 0
                except ArithmeticError:
                    R, L, P, r, d, st = np.zeros_like(A), np.zeros((m, m), np.uint32), [], 0, 0, -1
                out[pre + "meta"] = np.array([p, st, r, d], dtype=np.int64)
                out[pre + "A"] = A
                out[pre + "R"] = R
                out[pre + "L"] = L
                out[pre + "P"] = np.array(P, dtype=np.int64).reshape(-1, 2)
                names.append(pre)
    out["names"] = np.array(names)
    np.savez_compressed(os.path.join(HERE, fname), **out)
    print("%s: %d cases, %d LELA failures" % (fname, len(names),
                                              sum(int(out[n + "meta"][1] != 0) for n in names)))


def write_packed(fname):
    """Both packed forms of each input: prefix pk_..., A once, then for
    g = 0 (Elimination) and 1 (GaussJordan) meta<g> = [p, status, rank,
    det], E<g> and P<g>."""
    out = {}
    names = []
    for pi, p in enumerate(MODULI):
        for si, (m, n) in enumerate(SHAPES):
            for kind in range(3):
                if (m == 0 or n == 0) and kind:
                    continue
                A = case_matrix(1000 * pi + 10 * si + kind, m, n, p, kind)
                pre = "pk_%d_%d_%d_" % (pi, si, kind)
                out[pre + "A"] = A
                for g in (0, 1):
                    try:
                        E, P, r, d = oracle.ref_echelon_packed_L_zp(p, A, gauss_jordan=bool(g))
                        st = 0
                    except ArithmeticError:
                        E, P, r, d, st = np.zeros_like(A), [], 0, 0, -1
                    out[pre + "meta%d" % g] = np.array([p, st, r, d], dtype=np.int64)
                    out[pre + "E%d" % g] = E
                    out[pre + "P%d" % g] = np.array(P, dtype=np.int64).reshape(-1, 2)
                names.append(pre)
    out["names"] = np.array(names)
    np.savez_compressed(os.path.join(HERE, fname), **out)
    print("%s: %d inputs, %d LELA failures" % (fname, len(names),
                                               sum(int(out[n + "meta%d" % g][1] != 0)
                                                   for n in names for g in (0, 1))))


def main():
    assert oracle.have_ref(), "build oracle/_ref first (make -C oracle ref)"
    write(oracle.ref_echelon_reduced_L_zp, "transform_golden.npz")
    write(oracle.ref_gj_echelon_reduced_L_zp, "gj_transform_golden.npz")
    write_packed("packed_golden.npz")


if __name__ == "__main__":
    main()
