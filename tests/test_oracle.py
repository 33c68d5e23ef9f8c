"""Pinning the CPU oracle (the C restatement in oracle/lela_oracle.c):
(1) against the golden fixtures computed by LELA's own code, committed under
tests/golden/; (2) against LELA's own code live, where oracle/_ref was built
(randomised cases, including the error paths).  No GPU needed."""
import numpy as np
import pytest

import golden_io
import oracle
import props
from lela_b200 import gen

need_ref = pytest.mark.skipif(not oracle.have_ref(), reason="oracle/_ref (LELA's CPU code) not built")


def test_golden_gemm_small():
    for pre, p, a, b, A, B, C, R in golden_io.gemm_cases():
        assert np.array_equal(oracle.gemm_zp(p, A, B, C, a, b), R), pre


def test_golden_gemm_512():
    g = golden_io.data()[1]["gemm512"]
    p, n = g["p"], g["n"]
    A = gen.dense_zp(g["seeds"][0], n, n, p)
    B = gen.dense_zp(g["seeds"][1], n, n, p)
    C = gen.dense_zp(g["seeds"][2], n, n, p)
    assert golden_io.sha(A) == g["A"] and golden_io.sha(B) == g["B"] and golden_io.sha(C) == g["C"], \
        "input generator drifted"
    R = oracle.gemm_zp(p, A, B, C, 1, 1, threads=8)
    assert golden_io.sha(R) == g["R"]


def test_golden_trsm():
    for pre, p, upper, unit, a, bad, A, B, R in golden_io.trsm_cases():
        got, gbad = oracle.trsm_zp(p, A, B, upper, unit, a)
        assert gbad == bad, pre
        if bad is None:
            assert np.array_equal(got, R), pre


def test_golden_echelon():
    for pre, p, st, r, d, A, E in golden_io.echelon_cases():
        if st:
            with pytest.raises(ArithmeticError):
                oracle.echelon_zp(p, A)
            continue
        got, gr, gd = oracle.echelon_zp(p, A)
        assert (gr, gd) == (r, d), pre
        assert np.array_equal(got, E), pre


@pytest.mark.parametrize("unit", [False, True])
def test_golden_echelon_reduced(unit):
    for pre, p, st, r, d, A, E in golden_io.echelon_reduced_cases(unit):
        if st:
            with pytest.raises(ArithmeticError):
                oracle.echelon_reduced_zp(p, A, unit)
            continue
        got, gr, gd = oracle.echelon_reduced_zp(p, A, unit)
        assert (gr, gd) == (r, d), pre
        assert np.array_equal(got, E), pre


def test_golden_pluq():
    for pre, p, st, r, d, A, E, P, Q in golden_io.pluq_cases():
        if st:
            with pytest.raises(ArithmeticError):
                oracle.pluq_zp(p, A)
            continue
        got, gP, gQ, gr, gd = oracle.pluq_zp(p, A)
        assert (gr, gd) == (r, d) and gP == P and gQ == Q, pre
        assert np.array_equal(got, E), pre


def test_golden_transform():
    """Elimination::echelonize_reduced with compute_L: R, L, P, rank, det and
    LELA's failures, against LELA's own results."""
    n = 0
    for pre, p, st, r, d, A, R, L, P in golden_io.transform_cases():
        if st:
            with pytest.raises(ArithmeticError):
                oracle.echelon_reduced_L_zp(p, A)
            continue
        gR, gL, gP, gr, gd = oracle.echelon_reduced_L_zp(p, A)
        assert (gr, gd) == (r, d) and gP == P, pre
        assert np.array_equal(gR, R) and np.array_equal(gL, L), pre
        n += 1
    assert n >= 100


def test_golden_gj_transform():
    """GaussJordan::echelonize_reduced with its transform: R, L, P, rank, det
    and LELA's failures, against LELA's own results."""
    n = 0
    for pre, p, st, r, d, A, R, L, P in golden_io.transform_cases(gj=True):
        if st:
            with pytest.raises(ArithmeticError):
                oracle.gj_echelon_reduced_L_zp(p, A)
            continue
        if p >= 2 ** 31:
            continue  # LELA's wrapped inverses; the GPU form rejects such p
        gR, gL, gP, gr, gd = oracle.gj_echelon_reduced_L_zp(p, A)
        assert (gr, gd) == (r, d) and gP == P, pre
        assert np.array_equal(gR, R) and np.array_equal(gL, L), pre
        n += 1
    assert n >= 80


def test_gj_scaling_of_the_standard_transform():
    """The Python mirror's fast-method form: the standard transform with
    each pivot row scaled by its pivot, the pivots read from the fast
    method's reduced form, gives LELA's GaussJordan transform."""
    from lela_b200.api import scale_pivot_rows
    n = 0
    for pre, p, st, r, d, A, R, L, P in golden_io.transform_cases(gj=True):
        if st or p >= 2 ** 31:
            continue
        _, Le, Pe, re, de = oracle.echelon_reduced_L_zp(p, A)
        Rg, _, _ = oracle.echelon_reduced_zp(p, A)
        scale_pivot_rows(p, Le, Rg, re)
        assert np.array_equal(Le, L) and Pe == P and (re, de) == (r, d), pre
        n += 1
    assert n >= 80


def test_golden_packed_L():
    """Elimination::echelonize (default compute_L) and GaussJordan::
    echelonize: U with L below the diagonal, P, rank and det (GaussTransform's
    own d for GaussJordan), against LELA's own results."""
    n = 0
    for pre, gj, p, st, r, d, A, E, P in golden_io.packed_cases():
        if st:
            with pytest.raises(ArithmeticError):
                oracle.echelon_packed_L_zp(p, A, gj)
            continue
        if p >= 2 ** 31:
            continue
        gE, gP, gr, gd = oracle.echelon_packed_L_zp(p, A, gj)
        assert (gr, gd) == (r, d) and gP == P, (pre, gj)
        assert np.array_equal(gE, E), (pre, gj)
        n += 1
    assert n >= 160


def test_gauss_transform_det_from_pivots():
    """The Python mirror's determinant of GaussJordan::echelonize, computed
    from the pivot columns and values alone, equals LELA's."""
    from lela_b200.api import gauss_transform_det
    n = 0
    for pre, gj, p, st, r, d, A, E, P in golden_io.packed_cases():
        if st or not gj or p >= 2 ** 31:
            continue
        U, r2, _ = oracle.echelon_zp(p, A)
        pc = [int(np.flatnonzero(U[i])[0]) for i in range(r2)]
        assert gauss_transform_det(p, A.shape[1], pc, [int(U[i, c]) for i, c in enumerate(pc)]) == d, pre
        n += 1
    assert n >= 80


def test_packed_L_reference_property():
    """The property the reference's own tests check (tests/test-elimination.C:
    28-96): after Elimination::echelonize with compute_L, move_L
    (elimination.tcc:373-391) takes A's strictly lower entries into L = I,
    clearing them in A, and then L P A_in equals that A.  The same holds for
    GaussJordan::echelonize (tests/test-gauss-jordan.C:28-105)."""
    rng = np.random.default_rng(17)
    for p in (2, 251, 65521, 2147483647):
        for (m, n) in ((1, 1), (6, 9), (9, 6), (30, 30), (25, 60), (60, 25)):
            for kind in range(3):
                A = gen.dense_zp(int(rng.integers(1 << 30)), m, n, p)
                if kind == 1:
                    A[:, ::2] = 0
                elif kind == 2:
                    A[m // 3:] = (A[: m - m // 3] * 5) % p
                for gj in (False, True):
                    E, P, r, d = oracle.echelon_packed_L_zp(p, A, gj)
                    L = np.eye(m, dtype=object)
                    U = E.astype(object).copy()
                    for i in range(m):
                        for j in range(min(i, n)):
                            L[i, j] = U[i, j]
                            U[i, j] = 0
                    B = A.astype(object)
                    for a, b in P:
                        B[[a, b]] = B[[b, a]]
                    assert np.array_equal(L.dot(B) % p, U), (p, m, n, kind, gj)


def test_transform_identity():
    """R = L P A, with L = [[X, 0], [Y, I]] in the rank's blocks, and R the
    standard method's reduced form (p < 2^31, where Modular<uint32>'s
    inverse is exact)."""
    rng = np.random.default_rng(5)
    for p in (2, 251, 65521, 2147483647):
        for (m, n) in ((1, 1), (6, 9), (9, 6), (30, 30), (25, 60)):
            for kind in range(3):
                A = gen.dense_zp(int(rng.integers(1 << 30)), m, n, p)
                if kind == 1:
                    A[:, ::2] = 0
                elif kind == 2:
                    A[m // 3:] = (A[: m - m // 3] * 3) % p
                R, L, P, r, d = oracle.echelon_reduced_L_zp(p, A)
                B = A.astype(object)
                for a, b in P:
                    B[[a, b]] = B[[b, a]]
                assert np.array_equal((L.astype(object).dot(B) % p).astype(np.uint32), R)
                assert not L[:r, r:].any()
                assert np.array_equal(L[r:, r:], np.eye(m - r, dtype=np.uint32))
                R2, r2, d2 = oracle.echelon_reduced_zp(p, A, unit=True)
                assert np.array_equal(R, R2) and (r, d) == (r2, d2)


def test_golden_fl():
    for (pre, p, m, n, red, od, st, rank, det, rowptr, colidx, vals, R) in golden_io.fl_cases():
        got = oracle.fl_echelonize_zp(p, m, n, rowptr, colidx, vals, red, od)
        assert got["status"] == st, pre
        assert (got["rank"], got["det"]) == (rank, det), pre
        assert np.array_equal(got["R"], R), pre


def test_golden_fl_f4_digest():
    z, man = golden_io.data()
    X = gen.f4_matrix(7, 300, 65521, density=0.03)
    for pre in man["fl"]:
        if pre + "R_sha" not in man:
            continue
        assert golden_io.sha(np.concatenate([X.rowptr.view(np.uint32), X.colidx, X.vals])) == man[pre + "X_sha"]
        _, _, _, red, od, st, rank, det = (int(x) for x in z[pre + "meta"])
        got = oracle.fl_echelonize_zp(65521, X.m, X.n, X.rowptr, X.colidx, X.vals, red, od)
        assert (got["status"], got["rank"], got["det"]) == (st, rank, det), pre
        assert golden_io.sha(got["R"]) == man[pre + "R_sha"], pre


def test_golden_gf2():
    for pre, m, n, k, A, B, C, R in golden_io.gf2_gemm_cases():
        assert np.array_equal(oracle.gemm_gf2(A, B, C, k, n, 1, 1), R), pre
    for pre, m, n, r, A, E in golden_io.gf2_echelon_cases():
        got, gr = oracle.echelon_gf2(A, n)
        assert gr == r and np.array_equal(got, E), pre


def test_freivalds_catches_planted_error():
    """The property check used at full size rejects a result with one wrong
    entry (the mistake is planted in the oracle's own output, on the CPU)."""
    p = 65521
    A = gen.dense_zp(1, 64, 80, p); B = gen.dense_zp(2, 80, 50, p); C0 = gen.dense_zp(3, 64, 50, p)
    C = oracle.gemm_zp(p, A, B, C0, 1, 1)
    assert props.freivalds_gemm(p, A, B, C0, C, 1, 1)
    C[5, 7] = (C[5, 7] + 1) % p
    assert not props.freivalds_gemm(p, A, B, C0, C, 1, 1)


# ------------------------------------------------- live against LELA's code

@need_ref
@pytest.mark.parametrize("seed", range(4))
def test_live_gemm(seed):
    rng = np.random.default_rng(seed)
    for p in (251, 65521, 2147483647, 4294967291):
        m, n, k = (int(x) for x in rng.integers(1, 60, size=3))
        a, b = int(rng.integers(0, p)), int(rng.integers(0, p))
        A = gen.dense_zp(seed, m, k, p); B = gen.dense_zp(seed + 1, k, n, p); C = gen.dense_zp(seed + 2, m, n, p)
        assert np.array_equal(oracle.gemm_zp(p, A, B, C, a, b), oracle.ref_gemm_zp(p, A, B, C, a, b))


@need_ref
@pytest.mark.parametrize("seed", range(4))
def test_live_trsm(seed):
    rng = np.random.default_rng(100 + seed)
    for upper in (0, 1):
        for unit in (0, 1):
            p = int(rng.choice([251, 65521, 2147483647]))
            m, n = int(rng.integers(1, 70)), int(rng.integers(1, 20))
            U = gen.upper_zp(seed, m, p, unit=bool(unit))
            if not unit and m > 3 and seed % 2:
                U[m // 3, m // 3] = 0
            A = U if upper else np.ascontiguousarray(U.T)
            B = gen.dense_zp(seed + 5, m, n, p)
            a = int(rng.integers(0, p))
            r1, b1 = oracle.trsm_zp(p, A, B, upper, unit, a)
            r2, b2 = oracle.ref_trsm_zp(p, A, B, upper, unit, a)
            assert b1 == b2
            if b1 is None:
                assert np.array_equal(r1, r2)


def test_inverse_matches_lela_int_arithmetic():
    """Modular<uint32>::inv runs its Euclid in 32-bit ints: exact inverses
    below 2^31, and for p >= 2^31 the reference's wrapped result (here:
    failure for every tested unit)."""
    for p in (3, 251, 65521, 2147483647):
        for x in (1, 2, p - 1, 12345 % p or 1):
            y = oracle.inv_zp(p, x)
            assert y and (x * y) % p == 1
        assert oracle.inv_zp(p, 0) == 0
    assert oracle.inv_zp(65536, 2) == 0


@need_ref
def test_live_inverse_large_modulus():
    """p >= 2^31: whether LELA can invert a pivot decides whether the
    echelon form succeeds; the restatement must agree case by case."""
    for p in (2147483659, 4294967291):
        for seed in range(3):
            A = gen.dense_zp(seed, 6, 5, p)
            try:
                e2 = oracle.ref_echelon_zp(p, A, classical=True)
            except ArithmeticError:
                e2 = None
            try:
                e1 = oracle.echelon_zp(p, A)
            except ArithmeticError:
                e1 = None
            assert (e1 is None) == (e2 is None)
            if e1 is not None:
                assert np.array_equal(e1[0], e2[0]) and e1[1:] == e2[1:]


@need_ref
@pytest.mark.parametrize("seed", range(4))
def test_live_echelon(seed):
    p = [65521, 251, 2147483647, 3][seed]
    A = gen.dense_zp(seed, 45, 38, p)
    A[:, 5] = 0
    A[30:] = (A[:15] * 7) % p
    e1, r1, d1 = oracle.echelon_zp(p, A)
    e2, r2, d2 = oracle.ref_echelon_zp(p, A)
    e3, r3, d3 = oracle.ref_echelon_zp(p, A, classical=True)
    assert np.array_equal(e1, e2) and np.array_equal(e1, e3)
    assert (r1, d1) == (r2, d2) == (r3, d3)


@need_ref
@pytest.mark.parametrize("unit", [False, True])
@pytest.mark.parametrize("p", [2, 3, 251, 65521, 65536, 2147483647, 4294967291])
def test_live_echelon_reduced(p, unit):
    """GaussJordan::echelonize_reduced (unit: Elimination::echelonize_reduced)
    against the restatement: full rank,
    rank deficient (a product of thin factors), zero columns and rows, tall
    and wide, and LELA's pivot-inversion failures (composite p, p >= 2^31)."""
    rng = np.random.default_rng(p % 1000)
    for (m, n) in ((1, 1), (7, 13), (13, 7), (40, 40), (64, 100), (100, 64)):
        for kind in range(4):
            A = gen.dense_zp(int(rng.integers(1 << 30)), m, n, p)
            if kind == 1:
                A[:, ::3] = 0
            elif kind == 2:
                r = max(1, min(m, n) // 3)
                F = gen.dense_zp(1, m, r, p).astype(object) @ gen.dense_zp(2, r, n, p).astype(object)
                A = (F % p).astype(np.uint32)
            elif kind == 3:
                A[m // 2:] = 0
                A[:, :n // 2] = 0
            try:
                want = oracle.ref_echelon_reduced_zp(p, A, unit)
            except ArithmeticError:
                want = None
            try:
                got = oracle.echelon_reduced_zp(p, A, unit)
            except ArithmeticError:
                got = None
            assert (want is None) == (got is None), (m, n, kind)
            if want is not None:
                assert np.array_equal(got[0], want[0]) and got[1:] == want[1:], (m, n, kind)


@need_ref
@pytest.mark.parametrize("seed", range(6))
def test_live_fl(seed):
    p = 65521
    X = gen.f4_matrix_small(50 + seed, 50 + 10 * seed, 60 + 13 * seed, p, 0.08 + 0.02 * seed)
    for red, od in ((1, 0), (0, 0), (1, 1), (0, 1)):
        a = oracle.fl_echelonize_zp(p, X.m, X.n, X.rowptr, X.colidx, X.vals, red, od)
        b = oracle.ref_fl_echelonize_zp(p, X.m, X.n, X.rowptr, X.colidx, X.vals, red, od)
        assert (a["status"], a["rank"], a["det"]) == (b["status"], b["rank"], b["det"])
        assert np.array_equal(a["R"], b["R"])


@need_ref
def test_live_fl_wrong_form():
    """A row whose head lies left of the previous pivot: WrongMatrixForm."""
    p = 65521
    D = np.zeros((4, 6), dtype=np.uint32)
    D[0, 1] = 1; D[1, 3] = 1; D[2, 2] = 5; D[3, 4] = 1
    X = gen.CSR.from_dense(D)
    a = oracle.fl_echelonize_zp(p, X.m, X.n, X.rowptr, X.colidx, X.vals, 1, 0)
    b = oracle.ref_fl_echelonize_zp(p, X.m, X.n, X.rowptr, X.colidx, X.vals, 1, 0)
    assert a["status"] == b["status"] == 1
    assert a["bad_row"] == 2


@need_ref
def test_live_fl_f4_shaped():
    p = 65521
    X = gen.f4_matrix(3, 400, p, density=0.02)
    a = oracle.fl_echelonize_zp(p, X.m, X.n, X.rowptr, X.colidx, X.vals, 1, 0)
    b = oracle.ref_fl_echelonize_zp(p, X.m, X.n, X.rowptr, X.colidx, X.vals, 1, 0)
    assert (a["rank"], a["det"]) == (b["rank"], b["det"])
    assert np.array_equal(a["R"], b["R"])
    assert a["rank"] < X.m     # the planted dependencies lower the rank


@need_ref
@pytest.mark.parametrize("seed", range(3))
def test_live_gf2(seed):
    m, n, k = 40 + seed * 30, 70 + seed * 40, 65 + seed * 20
    A = gen.dense_gf2(seed, m, k); B = gen.dense_gf2(seed + 1, k, n); C = gen.dense_gf2(seed + 2, m, n)
    for a, b in ((1, 1), (1, 0), (0, 1)):
        assert np.array_equal(oracle.gemm_gf2(A, B, C, k, n, a, b), oracle.ref_gemm_gf2(A, B, C, k, n, a, b))
    E = gen.planted_rank_gf2(seed, m, n, min(m, n) // 2)
    e1, r1 = oracle.echelon_gf2(E, n)
    e2, r2 = oracle.ref_echelon_gf2(E, n)
    assert r1 == r2 and np.array_equal(e1, e2)


@need_ref
@pytest.mark.parametrize("p", [2, 3, 251, 65521, 65536, 2147483647, 4294967291])
def test_live_pluq(p):
    """Elimination::pluq against the restatement: L and U, both permutations,
    rank and det, on full-rank, rank-deficient, zero-column and zero-row
    inputs, and LELA's pivot-inversion failures."""
    rng = np.random.default_rng(p % 991)
    for (m, n) in ((1, 1), (7, 13), (13, 7), (40, 40), (48, 80), (80, 48)):
        for kind in range(4):
            A = gen.dense_zp(int(rng.integers(1 << 30)), m, n, p)
            if kind == 1:
                A[:, ::3] = 0
            elif kind == 2:
                r = max(1, min(m, n) // 3)
                F = gen.dense_zp(1, m, r, p).astype(object) @ gen.dense_zp(2, r, n, p).astype(object)
                A = (F % p).astype(np.uint32)
            elif kind == 3:
                A[m // 2:] = 0
                A[:, :n // 2] = 0
            try:
                want = oracle.ref_pluq_zp(p, A)
            except ArithmeticError:
                want = None
            try:
                got = oracle.pluq_zp(p, A)
            except ArithmeticError:
                got = None
            assert (want is None) == (got is None), (m, n, kind)
            if want is not None:
                assert np.array_equal(got[0], want[0]) and got[1:] == want[1:], (m, n, kind)


@need_ref
@pytest.mark.parametrize("p", [2, 3, 251, 65521, 65536, 2147483647, 4294967291])
def test_live_transform(p):
    """Elimination::echelonize_reduced (compute_L = true) against the
    restatement: R, L, P, rank and det on full-rank, rank-deficient,
    zero-column and zero-row inputs, and LELA's pivot-inversion failures."""
    rng = np.random.default_rng(p % 983)
    for (m, n) in ((1, 1), (2, 7), (7, 13), (13, 7), (40, 40), (48, 80), (80, 48)):
        for kind in range(4):
            A = gen.dense_zp(int(rng.integers(1 << 30)), m, n, p)
            if kind == 1:
                A[:, ::3] = 0
            elif kind == 2:
                r = max(1, min(m, n) // 3)
                F = gen.dense_zp(1, m, r, p).astype(object) @ gen.dense_zp(2, r, n, p).astype(object)
                A = (F % p).astype(np.uint32)
            elif kind == 3:
                A[m // 2:] = 0
                A[:, :n // 2] = 0
            try:
                want = oracle.ref_echelon_reduced_L_zp(p, A)
            except ArithmeticError:
                want = None
            try:
                got = oracle.echelon_reduced_L_zp(p, A)
            except ArithmeticError:
                got = None
            assert (want is None) == (got is None), (m, n, kind)
            if want is not None:
                assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1]), (m, n, kind)
                assert got[2:] == want[2:], (m, n, kind)


@need_ref
@pytest.mark.parametrize("p", [2, 3, 251, 65521, 65536, 2147483647, 4294967291])
def test_live_gj_transform(p):
    """GaussJordan::echelonize_reduced with its transform against the
    restatement (below 2^31; above it whether LELA fails must agree)."""
    rng = np.random.default_rng(p % 977)
    for (m, n) in ((1, 1), (2, 7), (7, 13), (13, 7), (40, 40), (48, 80), (80, 48)):
        for kind in range(4):
            A = gen.dense_zp(int(rng.integers(1 << 30)), m, n, p)
            if kind == 1:
                A[:, ::3] = 0
            elif kind == 2:
                r = max(1, min(m, n) // 3)
                F = gen.dense_zp(1, m, r, p).astype(object) @ gen.dense_zp(2, r, n, p).astype(object)
                A = (F % p).astype(np.uint32)
            elif kind == 3:
                A[m // 2:] = 0
                A[:, :n // 2] = 0
            try:
                want = oracle.ref_gj_echelon_reduced_L_zp(p, A)
            except ArithmeticError:
                want = None
            try:
                got = oracle.gj_echelon_reduced_L_zp(p, A)
            except ArithmeticError:
                got = None
            assert (want is None) == (got is None), (m, n, kind)
            if want is not None and p < 2 ** 31:
                assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1]), (m, n, kind)
                assert got[2:] == want[2:], (m, n, kind)


@need_ref
@pytest.mark.parametrize("p", [2, 3, 251, 65521, 65536, 2147483647, 4294967291])
def test_live_packed_L(p):
    """Both packed non-reduced forms against the restatement (below 2^31;
    above it whether LELA fails must agree)."""
    rng = np.random.default_rng(p % 971)
    for (m, n) in ((1, 1), (2, 7), (7, 13), (13, 7), (40, 40), (48, 80), (80, 48)):
        for kind in range(4):
            A = gen.dense_zp(int(rng.integers(1 << 30)), m, n, p)
            if kind == 1:
                A[:, ::3] = 0
            elif kind == 2:
                r = max(1, min(m, n) // 3)
                F = gen.dense_zp(1, m, r, p).astype(object) @ gen.dense_zp(2, r, n, p).astype(object)
                A = (F % p).astype(np.uint32)
            elif kind == 3:
                A[m // 2:] = 0
                A[:, :n // 2] = 0
            for gj in (False, True):
                try:
                    want = oracle.ref_echelon_packed_L_zp(p, A, gj)
                except ArithmeticError:
                    want = None
                try:
                    got = oracle.echelon_packed_L_zp(p, A, gj)
                except ArithmeticError:
                    got = None
                assert (want is None) == (got is None), (m, n, kind, gj)
                if want is not None and p < 2 ** 31:
                    assert np.array_equal(got[0], want[0]) and got[1:] == want[1:], (m, n, kind, gj)
