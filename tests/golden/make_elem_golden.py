"""Generate tests/golden/elem_golden.npz from LELA's own CPU code: BLAS3::gemm
and BLAS3::trsm over Modular<uint8>, Modular<uint16>, Modular<float> and
Modular<double> (the element types of tests/test-blas-zp-module.C:161-168,
with its moduli 251, 65521, 2039, 4093, 33554393, 67108859, plus an even
modulus for float and double), through oracle/_ref/liblela_ref.so.

    python tests/golden/make_elem_golden.py

Inputs are seeded uniform residues (lela_b200.gen.dense_zp) stored in each
type's representation; the outputs are what LELA computes.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from lela_b200 import gen  # noqa: E402

CASES = [(np.uint8, 251), (np.uint16, 65521), (np.float32, 2039), (np.float32, 4093),
         (np.float32, 10), (np.float64, 33554393), (np.float64, 67108859), (np.float64, 1000)]


def main():
    assert oracle.have_ref(), "build oracle/_ref first (make -C oracle ref)"
    out = {}
    for ci, (dt, p) in enumerate(CASES):
        rep = lambda R: oracle.from_residues(R, p, dt)
        # gemm: C <- a A B + b C, the reference test's 50 x 50 by 50 x 30
        # shape and two others
        for gi, (m, n, k, a, b) in enumerate([(50, 30, 50, 1, 1), (17, 33, 70, p - 1, 3 % p),
                                              (12, 7, 5, 5 % p, 0)]):
            A = rep(gen.dense_zp(100 * ci + 3 * gi, m, k, p))
            B = rep(gen.dense_zp(100 * ci + 3 * gi + 1, k, n, p))
            C = rep(gen.dense_zp(100 * ci + 3 * gi + 2, m, n, p))
            R = oracle.ref_gemm_zp_elem(p, A, B, C, a, b)
            pre = "gemm_%d_%d_" % (ci, gi)
            out.update({pre + "A": A, pre + "B": B, pre + "C": C, pre + "R": R,
                        pre + "meta": np.array([p, a, b], dtype=np.uint64)})
        # trsm: B <- a A^-1 B, upper / lower, unit / general diagonal; the
        # general ones with a zero planted on the diagonal in one case
        ti = 0
        for upper in (0, 1):
            for unit in (0, 1):
                for sing in ((0, 1) if not unit else (0,)):
                    m, n = 24, 9
                    L = gen.dense_zp(100 * ci + 50 + ti, m, m, p)
                    L = np.triu(L) if upper else np.tril(L)
                    if unit:
                        np.fill_diagonal(L, 1)
                    else:
                        d = np.diag(L).copy()
                        d[d == 0] = 1
                        if sing:
                            d[17] = 0
                        np.fill_diagonal(L, d)
                    A = rep(L)
                    B = rep(gen.dense_zp(100 * ci + 70 + ti, m, n, p))
                    a = 3 % p
                    R, bad = oracle.ref_trsm_zp_elem(p, A, B, upper, unit, a)
                    pre = "trsm_%d_%d_" % (ci, ti)
                    out.update({pre + "A": A, pre + "B": B, pre + "R": R,
                                pre + "meta": np.array([p, a, upper, unit,
                                                        -1 if bad is None else bad], dtype=np.int64)})
                    ti += 1
    np.savez_compressed(os.path.join(HERE, "elem_golden.npz"), **out)
    print("wrote", len(out), "arrays")


if __name__ == "__main__":
    main()
