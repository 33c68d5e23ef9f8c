"""Generate the golden fixtures of tests/golden/ from LELA's own CPU code.

    python tests/golden/make_golden.py

Needs oracle/_ref/liblela_ref.so (built by `make -C oracle ref` from the
reference sources).  Inputs come from lela_b200.gen (seeded); outputs are
what LELA itself computes: BLAS3::gemm, BLAS3::trsm, the dense echelon forms
of EchelonForm (GaussJordan + move_L; reduced: GaussJordan::
echelonize_reduced and Elimination::echelonize_reduced), Elimination::pluq,
FaugereLachartre::echelonize in all
four modes, and the GF(2) gemm / echelon form.  Small cases store inputs
and outputs; the larger ones store SHA-256 digests of inputs and outputs.
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from lela_b200 import gen  # noqa: E402


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main():
    assert oracle.have_ref(), "build oracle/_ref first (make -C oracle ref)"
    out = {}
    manifest = {}

    # ---- Z/p gemm, small, every limb count and coefficient pattern
    cases = []
    for i, (p, m, n, k, a, b) in enumerate([
            (251, 24, 17, 33, 1, 1), (65521, 24, 17, 33, 65520, 1), (65521, 9, 31, 70, 3, 0),
            (2147483647, 20, 20, 40, 7, 11), (4294967291, 13, 29, 21, 0, 5), (2, 30, 30, 64, 1, 1)]):
        A = gen.dense_zp(10 * i, m, k, p)
        B = gen.dense_zp(10 * i + 1, k, n, p)
        C = gen.dense_zp(10 * i + 2, m, n, p)
        R = oracle.ref_gemm_zp(p, A, B, C, a, b, module=0)
        R2 = oracle.ref_gemm_zp(p, A, B, C, a, b, module=1)
        assert np.array_equal(R, R2)
        pre = "gemm%d_" % i
        out.update({pre + "A": A, pre + "B": B, pre + "C": C, pre + "R": R,
                    pre + "meta": np.array([p, a, b], dtype=np.uint64)})
        cases.append(pre)
    manifest["gemm_small"] = cases

    # ---- Z/p gemm, the plain 512^3 case (p = 65521, seed 0), digests only
    p, n = 65521, 512
    A = gen.dense_zp(0, n, n, p)
    B = gen.dense_zp(1, n, n, p)
    C = gen.dense_zp(2, n, n, p)
    R = oracle.ref_gemm_zp(p, A, B, C, 1, 1, module=0)
    manifest["gemm512"] = {"p": p, "n": n, "seeds": [0, 1, 2], "A": sha(A), "B": sha(B), "C": sha(C),
                           "R": sha(R), "R_corner": R[:4, :4].tolist()}

    # ---- Z/p trsm
    cases = []
    ci = 0
    for upper in (0, 1):
        for unit in (0, 1):
            for a in (1, 5):
                m, nn, p = 37, 11, 65521
                U = gen.upper_zp(100 + ci, m, p, unit=bool(unit))
                A = U if upper else np.ascontiguousarray(U.T)
                B = gen.dense_zp(200 + ci, m, nn, p)
                R, bad = oracle.ref_trsm_zp(p, A, B, upper, unit, a)
                pre = "trsm%d_" % ci
                out.update({pre + "A": A, pre + "B": B, pre + "R": R,
                            pre + "meta": np.array([p, upper, unit, a, -1 if bad is None else bad],
                                                   dtype=np.int64)})
                cases.append(pre)
                ci += 1
    # singular diagonals: LELA reports the first one its recursion meets
    for upper in (0, 1):
        p = 2147483647
        U = gen.upper_zp(300 + upper, 40, p)
        U[7, 7] = 0
        U[29, 29] = 0
        A = U if upper else np.ascontiguousarray(U.T)
        B = gen.dense_zp(400 + upper, 40, 6, p)
        R, bad = oracle.ref_trsm_zp(p, A, B, upper, 0, 1)
        pre = "trsm%d_" % ci
        out.update({pre + "A": A, pre + "B": B, pre + "R": R,
                    pre + "meta": np.array([p, upper, 0, 1, bad], dtype=np.int64)})
        cases.append(pre)
        ci += 1
    manifest["trsm"] = cases

    # ---- dense echelon form (non-reduced, LELA's pivot rule)
    cases = []
    for i, (p, m, nn) in enumerate([(65521, 30, 40), (65521, 50, 30), (251, 40, 40),
                                    (2147483647, 33, 57), (4294967291, 20, 25)]):
        A = gen.dense_zp(500 + i, m, nn, p)
        A[:, 3] = 0
        if m > 20:
            A[m - 8:] = (A[:8] * 3) % p     # rank deficiency
        A[2] = 0                            # zero row
        try:
            E, r, d = oracle.ref_echelon_zp(p, A)
            st = 0
        except ArithmeticError:     # LELA cannot invert a pivot (p >= 2^31)
            E, r, d, st = A, 0, 0, 1
        pre = "ech%d_" % i
        out.update({pre + "A": A, pre + "E": E, pre + "meta": np.array([p, st, r, d], dtype=np.uint64)})
        cases.append(pre)
    manifest["echelon"] = cases

    # ---- dense reduced echelon form (EchelonForm::echelonize (A, true):
    #      GaussJordan::echelonize_reduced)
    cases, units = [], []
    for i, (p, m, nn) in enumerate([(65521, 30, 40), (65521, 50, 30), (251, 40, 40), (2, 24, 70),
                                    (65536, 12, 12), (2147483647, 33, 57), (4294967291, 20, 25),
                                    (65521, 70, 9)]):
        A = gen.dense_zp(600 + i, m, nn, p)
        A[:, 3 % nn] = 0
        if m > 20:
            A[m - 8:] = (A[:8] * 3) % p     # rank deficiency
        A[2] = 0                            # zero row
        try:
            E, r, d = oracle.ref_echelon_reduced_zp(p, A)
            st = 0
        except ArithmeticError:     # LELA cannot invert a pivot
            E, r, d, st = A, 0, 0, 1
        pre = "rech%d_" % i
        out.update({pre + "A": A, pre + "E": E, pre + "meta": np.array([p, st, r, d], dtype=np.uint64)})
        cases.append(pre)
        # the standard method's reduced form (Elimination::echelonize_reduced,
        # pivots scaled to 1) of the same input
        try:
            E, r, d = oracle.ref_echelon_reduced_zp(p, A, unit=True)
            st = 0
        except ArithmeticError:
            E, r, d, st = A, 0, 0, 1
        pre = "rechu%d_" % i
        out.update({pre + "A": A, pre + "E": E, pre + "meta": np.array([p, st, r, d], dtype=np.uint64)})
        units.append(pre)
    manifest["echelon_reduced"] = cases
    manifest["echelon_reduced_unit"] = units

    # ---- PLUQ decomposition (Elimination::pluq)
    cases = []
    for i, (p, m, nn) in enumerate([(65521, 20, 30), (65521, 30, 20), (251, 25, 25), (2, 18, 40),
                                    (65536, 10, 10), (2147483647, 16, 24)]):
        A = gen.dense_zp(700 + i, m, nn, p)
        A[:, 2] = 0
        A[m - 4:] = (A[:4] * 5) % p       # rank deficiency
        try:
            E, P, Q, r, d = oracle.ref_pluq_zp(p, A)
            st = 0
        except ArithmeticError:
            E, P, Q, r, d, st = A, [], [], 0, 0, 1
        pre = "pluq%d_" % i
        out.update({pre + "A": A, pre + "E": E, pre + "P": np.array(P, dtype=np.int64).reshape(-1, 2),
                    pre + "Q": np.array(Q, dtype=np.int64).reshape(-1, 2),
                    pre + "meta": np.array([p, st, r, d], dtype=np.uint64)})
        cases.append(pre)
    manifest["pluq"] = cases

    # ---- Faugere-Lachartre, the reference test's matrix family and an
    #      F4-shaped matrix
    cases = []
    fl_inputs = [("small", s, gen.f4_matrix_small(s, mm, nn, 65521, 0.1))
                 for s, (mm, nn) in enumerate([(60, 70), (96, 128), (40, 90)])]
    fl_inputs.append(("f4", 7, gen.f4_matrix(7, 300, 65521, density=0.03)))
    for j, (kind, seed, X) in enumerate(fl_inputs):
        for red, od in ((1, 0), (0, 0), (1, 1), (0, 1)):
            r = oracle.ref_fl_echelonize_zp(65521, X.m, X.n, X.rowptr, X.colidx, X.vals, red, od)
            pre = "fl%d_%d%d_" % (j, red, od)
            out.update({pre + "meta": np.array([65521, X.m, X.n, red, od, r["status"], r["rank"],
                                                 r["det"]], dtype=np.uint64)})
            if kind == "small":
                out.update({pre + "rowptr": X.rowptr, pre + "colidx": X.colidx, pre + "vals": X.vals,
                            pre + "R": r["R"]})
            else:
                manifest[pre + "R_sha"] = sha(r["R"])
                manifest[pre + "R_shape"] = list(r["R"].shape)
                manifest[pre + "X_sha"] = sha(np.concatenate([X.rowptr.view(np.uint32), X.colidx, X.vals]))
            cases.append(pre)
    manifest["fl"] = cases

    # ---- GF(2)
    cases = []
    for i, (m, nn, k) in enumerate([(70, 130, 65), (64, 64, 64), (5, 200, 129)]):
        A = gen.dense_gf2(700 + i, m, k)
        B = gen.dense_gf2(710 + i, k, nn)
        C = gen.dense_gf2(720 + i, m, nn)
        R = oracle.ref_gemm_gf2(A, B, C, k, nn, 1, 1)
        pre = "g2mm%d_" % i
        out.update({pre + "A": A, pre + "B": B, pre + "C": C, pre + "R": R,
                    pre + "meta": np.array([m, nn, k], dtype=np.uint64)})
        cases.append(pre)
    manifest["gf2_gemm"] = cases
    cases = []
    for i, (m, nn, r) in enumerate([(100, 90, 40), (64, 200, 64), (130, 70, 70)]):
        A = gen.planted_rank_gf2(800 + i, m, nn, r)
        E, rk = oracle.ref_echelon_gf2(A, nn)
        pre = "g2ech%d_" % i
        out.update({pre + "A": A, pre + "E": E, pre + "meta": np.array([m, nn, rk], dtype=np.uint64)})
        cases.append(pre)
    manifest["gf2_echelon"] = cases

    np.savez_compressed(os.path.join(HERE, "lela_golden.npz"), **out)
    with open(os.path.join(HERE, "lela_golden.json"), "w") as f:
        json.dump(manifest, f, indent=1, sort_keys=True)
    print("wrote", len(out), "arrays")


if __name__ == "__main__":
    main()
