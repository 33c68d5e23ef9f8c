"""CPU checkers for the LELA hot path -- TEST INFRASTRUCTURE ONLY.

Two libraries sit behind this module:

* ``oracle/liboracle.so`` -- the plain-C restatement in ``lela_oracle.c``
  (every function cites the LELA routine it restates);
* ``oracle/_ref/liblela_ref.so`` -- LELA's own CPU code, compiled from the
  unmodified reference sources by ``oracle/Makefile`` (present only where the
  reference tree was available at build time, or where the prebuilt file was
  carried along).

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package, and only as the checker.  The product
(``lela_b200``) never imports it.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_P = ctypes.c_void_p
_S = ctypes.c_size_t
_U = ctypes.c_uint32
_I = ctypes.c_int

_lib = None
_ref = None


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def lib():
    """The C restatement (liboracle.so); built on first use if missing."""
    global _lib
    if _lib is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            import subprocess
            subprocess.run(["make", "-C", _HERE, "liboracle.so"], check=True,
                           stdout=subprocess.DEVNULL)
        L = ctypes.CDLL(path)
        L.oracle_gemm_zp_u32.argtypes = [_U, _S, _S, _S, _U, _P, _S, _P, _S, _U, _P, _S]
        L.oracle_gemm_zp_u32_threads.argtypes = [_I, _U, _S, _S, _S, _U, _P, _S, _P, _S, _U, _P, _S]
        L.oracle_trsm_zp_u32.argtypes = [_U, _I, _I, _S, _S, _U, _P, _S, _P, _S, ctypes.POINTER(_S)]
        L.oracle_echelon_zp_u32.argtypes = [_U, _S, _S, _P, _S, ctypes.POINTER(_S), ctypes.POINTER(_U)]
        L.oracle_echelon_reduced_zp_u32.argtypes = [_U, _S, _S, _P, _S, ctypes.POINTER(_S),
                                                    ctypes.POINTER(_U)]
        L.oracle_echelon_reduced_unit_zp_u32.argtypes = [_U, _S, _S, _P, _S, ctypes.POINTER(_S),
                                                         ctypes.POINTER(_U)]
        L.oracle_fl_echelonize_zp_u32.argtypes = [_U, _S, _S, _P, _P, _P, _I, _I, _P, _S,
                                                  ctypes.POINTER(_S), ctypes.POINTER(_U),
                                                  ctypes.POINTER(_S), ctypes.POINTER(_S)]
        L.oracle_gemm_gf2.argtypes = [_S, _S, _S, _I, _P, _S, _P, _S, _I, _P, _S]
        L.oracle_echelon_gf2.argtypes = [_S, _S, _P, _S, ctypes.POINTER(_S)]
        L.oracle_pluq_zp_u32.argtypes = [_U, _S, _S, _P, _S, _P, ctypes.POINTER(_S), _P, ctypes.POINTER(_S),
                                         ctypes.POINTER(_S), ctypes.POINTER(_U)]
        L.oracle_echelon_reduced_L_zp_u32.argtypes = [_U, _S, _S, _P, _S, _P, _S, _P, ctypes.POINTER(_S),
                                                      ctypes.POINTER(_S), ctypes.POINTER(_U)]
        L.oracle_gj_echelon_reduced_L_zp_u32.argtypes = [_U, _S, _S, _P, _S, _P, _S, _P, ctypes.POINTER(_S),
                                                         ctypes.POINTER(_S), ctypes.POINTER(_U)]
        L.oracle_echelon_packed_L_zp_u32.argtypes = [_I, _U, _S, _S, _P, _S, _P, ctypes.POINTER(_S),
                                                     ctypes.POINTER(_S), ctypes.POINTER(_U)]
        L.oracle_inv_zp.argtypes = [_U, _U]
        L.oracle_inv_zp.restype = _U
        _lib = L
    return _lib


def ref_path():
    return os.path.join(_HERE, "_ref", "liblela_ref.so")


def have_ref():
    return os.path.exists(ref_path())


def ref():
    """LELA's own CPU code (oracle/_ref/liblela_ref.so), or None."""
    global _ref
    if _ref is None and have_ref():
        L = ctypes.CDLL(ref_path())
        L.lela_ref_gemm_zp_u32.argtypes = [_I, _U, _S, _S, _S, _U, _P, _S, _P, _S, _U, _P, _S]
        L.lela_ref_gemm_zp_u32_threads.argtypes = [_I, _U, _S, _S, _S, _U, _P, _S, _P, _S, _U, _P, _S]
        L.lela_ref_trsm_zp_u32.argtypes = [_U, _I, _I, _S, _S, _U, _P, _S, _P, _S, ctypes.POINTER(_S)]
        L.lela_ref_trsm_zp_u32_threads.argtypes = [_I, _U, _I, _I, _S, _S, _U, _P, _S, _P, _S]
        L.lela_ref_echelon_zp_u32.argtypes = [_U, _S, _S, _P, _S, ctypes.POINTER(_S), ctypes.POINTER(_U)]
        L.lela_ref_echelon_reduced_zp_u32.argtypes = [_U, _S, _S, _P, _S, ctypes.POINTER(_S),
                                                      ctypes.POINTER(_U)]
        L.lela_ref_elim_echelon_reduced_zp_u32.argtypes = [_U, _S, _S, _P, _S, ctypes.POINTER(_S),
                                                           ctypes.POINTER(_U)]
        L.lela_ref_elim_echelon_zp_u32.argtypes = [_U, _S, _S, _P, _S, ctypes.POINTER(_S), ctypes.POINTER(_U)]
        L.lela_ref_fl_echelonize_zp_u32.argtypes = [_U, _S, _S, _P, _P, _P, _I, _I, _P, _S,
                                                    ctypes.POINTER(_S), ctypes.POINTER(_U), ctypes.POINTER(_S)]
        L.lela_ref_gemm_gf2.argtypes = [_S, _S, _S, _I, _P, _S, _P, _S, _I, _P, _S]
        L.lela_ref_echelon_gf2.argtypes = [_S, _S, _P, _S, ctypes.POINTER(_S)]
        L.lela_ref_detect_format.argtypes = [ctypes.c_char_p]
        L.lela_ref_read_dumas.argtypes = [_U, ctypes.c_char_p, _S, ctypes.POINTER(_S), ctypes.POINTER(_S), _P]
        L.lela_ref_write_dumas.argtypes = [_U, _S, _S, _P, _S, ctypes.c_char_p, _S, ctypes.POINTER(_S)]
        L.lela_ref_write_matrix.argtypes = [_I, _U, _S, _S, _P, _S, ctypes.c_char_p, _S, ctypes.POINTER(_S)]
        L.lela_ref_read_matrix.argtypes = [_I, _U, ctypes.c_char_p, _S, _S, _P]
        L.lela_ref_gemm_zp_elem.argtypes = [_I, _U, _S, _S, _S, _U, _P, _S, _P, _S, _U, _P, _S]
        L.lela_ref_trsm_zp_elem.argtypes = [_I, _U, _I, _I, _S, _S, _U, _P, _S, _P, _S, ctypes.POINTER(_S)]
        L.lela_ref_pluq_zp_u32.argtypes = [_U, _S, _S, _P, _S, _P, ctypes.POINTER(_S), _P, ctypes.POINTER(_S),
                                           ctypes.POINTER(_S), ctypes.POINTER(_U)]
        L.lela_ref_elim_echelon_reduced_L_zp_u32.argtypes = [_U, _S, _S, _P, _S, _P, _S, _P,
                                                             ctypes.POINTER(_S), ctypes.POINTER(_S),
                                                             ctypes.POINTER(_U)]
        L.lela_ref_gj_echelon_reduced_L_zp_u32.argtypes = [_U, _S, _S, _P, _S, _P, _S, _P,
                                                           ctypes.POINTER(_S), ctypes.POINTER(_S),
                                                           ctypes.POINTER(_U)]
        L.lela_ref_echelon_packed_L_zp_u32.argtypes = [_I, _U, _S, _S, _P, _S, _P, ctypes.POINTER(_S),
                                                       ctypes.POINTER(_S), ctypes.POINTER(_U)]
        _ref = L
    return _ref


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


# ------------------------------------------------------------- restatement --

def gemm_zp(p, A, B, C, a=1, b=1, threads=1):
    A = _c(A, np.uint32); B = _c(B, np.uint32); C = _c(C, np.uint32).copy()
    m, k = A.shape; n = B.shape[1]
    if threads > 1:
        lib().oracle_gemm_zp_u32_threads(threads, p, m, n, k, a, _ptr(A), k, _ptr(B), n, b, _ptr(C), n)
    else:
        lib().oracle_gemm_zp_u32(p, m, n, k, a, _ptr(A), k, _ptr(B), n, b, _ptr(C), n)
    return C


def trsm_zp(p, A, B, upper, diag_is_one, a=1):
    """Returns (B', bad_idx or None)."""
    A = _c(A, np.uint32); B = _c(B, np.uint32).copy()
    m = A.shape[0]; n = B.shape[1]
    bad = _S(0)
    rc = lib().oracle_trsm_zp_u32(p, int(upper), int(diag_is_one), m, n, a, _ptr(A), m, _ptr(B), n, ctypes.byref(bad))
    return B, (bad.value if rc else None)


# Other Modular<T> element types (lela/ring/modular.h:115-330): uint8 and
# uint16 hold residues 0 .. p-1, float and double the symmetric
# representative (ModularTraits<float>::reduce: fmod, then shift_up v < -p/2
# -> v + p, then shift_down v > p/2 -> v - p).  Their gemm and trsm are exact
# Z/p arithmetic (lela/blas/level3-modular.tcc:25-122 keeps every partial sum
# below the mantissa), so the restatement runs the uint32 restatement on the
# residues and stores the result in the type's representation.
ELEM_CODES = {np.dtype(np.uint8): 1, np.dtype(np.uint16): 2, np.dtype(np.float32): 5,
              np.dtype(np.float64): 6}


def to_residues(X, p):
    """Elements of Modular<T> (T = X.dtype) as uint32 residues."""
    X = np.asarray(X)
    if X.dtype.kind == "f":
        v = X.astype(np.int64)
        return np.where(v < 0, v + p, v).astype(np.uint32)
    return X.astype(np.uint32)


def from_residues(R, p, dtype):
    """uint32 residues as elements of Modular<dtype> (for float / double the
    representative in [-p/2, p/2]; +p/2 for the residue p/2 of an even p)."""
    dtype = np.dtype(dtype)
    R = np.asarray(R, dtype=np.int64)
    if dtype.kind == "f":
        return np.where(2 * R > p, R - p, R).astype(dtype)
    return R.astype(dtype)


def gemm_zp_elem(p, A, B, C, a=1, b=1):
    dt = np.asarray(C).dtype
    R = gemm_zp(p, to_residues(A, p), to_residues(B, p), to_residues(C, p), a, b)
    return from_residues(R, p, dt)


def trsm_zp_elem(p, A, B, upper, diag_is_one, a=1):
    """Returns (B', bad_idx or None)."""
    dt = np.asarray(B).dtype
    R, bad = trsm_zp(p, to_residues(A, p), to_residues(B, p), upper, diag_is_one, a)
    return from_residues(R, p, dt), bad


def echelon_zp(p, A):
    A = _c(A, np.uint32).copy()
    m, n = A.shape
    r = _S(0); d = _U(0)
    rc = lib().oracle_echelon_zp_u32(p, m, n, _ptr(A), n, ctypes.byref(r), ctypes.byref(d))
    if rc:
        raise ArithmeticError("pivot not invertible")
    return A, r.value, d.value


def echelon_reduced_zp(p, A, unit=False):
    """unit: the standard method's form (pivots 1)."""
    A = _c(A, np.uint32).copy()
    m, n = A.shape
    r = _S(0); d = _U(0)
    fn = lib().oracle_echelon_reduced_unit_zp_u32 if unit else lib().oracle_echelon_reduced_zp_u32
    rc = fn(p, m, n, _ptr(A), n, ctypes.byref(r), ctypes.byref(d))
    if rc:
        raise ArithmeticError("pivot not invertible")
    return A, r.value, d.value


def _pluq(fn, p, A):
    A = _c(A, np.uint32).copy()
    m, n = A.shape
    k = max(min(m, n), 1)
    P = np.zeros(2 * k, dtype=np.uint64); Q = np.zeros(2 * k, dtype=np.uint64)
    np_ = _S(0); nq = _S(0); r = _S(0); d = _U(0)
    if fn(p, m, n, _ptr(A), max(n, 1), _ptr(P), ctypes.byref(np_), _ptr(Q), ctypes.byref(nq),
          ctypes.byref(r), ctypes.byref(d)):
        raise ArithmeticError("pivot not invertible")
    pairs = lambda X, c: [(int(X[2 * t]), int(X[2 * t + 1])) for t in range(c)]
    return A, pairs(P, np_.value), pairs(Q, nq.value), r.value, d.value


def pluq_zp(p, A):
    """Elimination::pluq restated: (LU in place, P, Q, rank, det)."""
    return _pluq(lib().oracle_pluq_zp_u32, p, A)


def _echelon_L(fn, p, A):
    A = _c(A, np.uint32).copy()
    m, n = A.shape
    L = np.zeros((m, m), dtype=np.uint32)
    P = np.zeros(2 * max(min(m, n), 1), dtype=np.uint64)
    np_ = _S(0); r = _S(0); d = _U(0)
    if fn(p, m, n, _ptr(A), max(n, 1), _ptr(L), max(m, 1), _ptr(P), ctypes.byref(np_),
          ctypes.byref(r), ctypes.byref(d)):
        raise ArithmeticError("pivot not invertible")
    return A, L, [(int(P[2 * t]), int(P[2 * t + 1])) for t in range(np_.value)], r.value, d.value


def echelon_reduced_L_zp(p, A):
    """Elimination::echelonize_reduced with compute_L, restated:
    (R, L, P, rank, det) with R = L P A."""
    return _echelon_L(lib().oracle_echelon_reduced_L_zp_u32, p, A)


def _packed(fn, gj, p, A):
    A = _c(A, np.uint32).copy()
    m, n = A.shape
    P = np.zeros(2 * max(min(m, n), 1), dtype=np.uint64)
    np_ = _S(0); r = _S(0); d = _U(0)
    if fn(gj, p, m, n, _ptr(A), max(n, 1), _ptr(P), ctypes.byref(np_), ctypes.byref(r), ctypes.byref(d)):
        raise ArithmeticError("pivot not invertible")
    return A, [(int(P[2 * t]), int(P[2 * t + 1])) for t in range(np_.value)], r.value, d.value


def echelon_packed_L_zp(p, A, gauss_jordan=False):
    """Elimination::echelonize (gauss_jordan: GaussJordan::echelonize) with
    L kept below the diagonal, restated: (A, P, rank, det)."""
    return _packed(lib().oracle_echelon_packed_L_zp_u32, int(gauss_jordan), p, A)


def gj_echelon_reduced_L_zp(p, A):
    """GaussJordan::echelonize_reduced with its transform, restated:
    (R, L, P, rank, det) with R = L P A, pivots keeping their values."""
    return _echelon_L(lib().oracle_gj_echelon_reduced_L_zp_u32, p, A)


def fl_echelonize_zp(p, m, n, rowptr, colidx, vals, reduced=True, only_D=False):
    """Returns dict(status, R (rows x n), rank, det, bad_row)."""
    rowptr = _c(rowptr, np.uint64); colidx = _c(colidx, np.uint32); vals = _c(vals, np.uint32)
    R = np.zeros((max(m, 1), n), dtype=np.uint32)
    rk = _S(0); det = _U(0); rows = _S(0); bad = _S(0)
    st = lib().oracle_fl_echelonize_zp_u32(p, m, n, _ptr(rowptr), _ptr(colidx), _ptr(vals),
                                           int(reduced), int(only_D), _ptr(R), n,
                                           ctypes.byref(rk), ctypes.byref(det), ctypes.byref(rows),
                                           ctypes.byref(bad))
    return dict(status=st, R=R[:rows.value] if st == 0 else None, rank=rk.value, det=det.value,
                bad_row=bad.value)


def gemm_gf2(A, B, C, k, n, a=1, b=1):
    A = _c(A, np.uint64); B = _c(B, np.uint64); C = _c(C, np.uint64).copy()
    m = A.shape[0]
    lib().oracle_gemm_gf2(m, n, k, a, _ptr(A), A.shape[1], _ptr(B), B.shape[1], b, _ptr(C), C.shape[1])
    return C


def echelon_gf2(A, n):
    A = _c(A, np.uint64).copy()
    r = _S(0)
    lib().oracle_echelon_gf2(A.shape[0], n, _ptr(A), A.shape[1], ctypes.byref(r))
    return A, r.value


def inv_zp(p, x):
    return lib().oracle_inv_zp(p, x)


# ------------------------------------------------------- LELA's own code --

def ref_gemm_zp(p, A, B, C, a=1, b=1, module=0, threads=1):
    A = _c(A, np.uint32); B = _c(B, np.uint32); C = _c(C, np.uint32).copy()
    m, k = A.shape; n = B.shape[1]
    if threads > 1:
        ref().lela_ref_gemm_zp_u32_threads(threads, p, m, n, k, a, _ptr(A), k, _ptr(B), n, b, _ptr(C), n)
    else:
        ref().lela_ref_gemm_zp_u32(module, p, m, n, k, a, _ptr(A), k, _ptr(B), n, b, _ptr(C), n)
    return C


def ref_trsm_zp(p, A, B, upper, diag_is_one, a=1, threads=1):
    A = _c(A, np.uint32); B = _c(B, np.uint32).copy()
    m = A.shape[0]; n = B.shape[1]
    if threads > 1:
        ref().lela_ref_trsm_zp_u32_threads(threads, p, int(upper), int(diag_is_one), m, n, a,
                                           _ptr(A), m, _ptr(B), n)
        return B, None
    bad = _S(0)
    rc = ref().lela_ref_trsm_zp_u32(p, int(upper), int(diag_is_one), m, n, a, _ptr(A), m, _ptr(B), n, ctypes.byref(bad))
    return B, (bad.value if rc else None)


def ref_gemm_zp_elem(p, A, B, C, a=1, b=1):
    """LELA's BLAS3::gemm on Context<Modular<T> >, T = the arrays' dtype."""
    dt = np.asarray(C).dtype
    A = _c(A, dt); B = _c(B, dt); C = _c(C, dt).copy()
    m, k = A.shape; n = B.shape[1]
    rc = ref().lela_ref_gemm_zp_elem(ELEM_CODES[dt], p, m, n, k, a, _ptr(A), k, _ptr(B), n, b, _ptr(C), n)
    assert rc == 0, rc
    return C


def ref_trsm_zp_elem(p, A, B, upper, diag_is_one, a=1):
    dt = np.asarray(B).dtype
    A = _c(A, dt); B = _c(B, dt).copy()
    m = A.shape[0]; n = B.shape[1]
    bad = _S(0)
    rc = ref().lela_ref_trsm_zp_elem(ELEM_CODES[dt], p, int(upper), int(diag_is_one), m, n, a,
                                     _ptr(A), m, _ptr(B), n, ctypes.byref(bad))
    assert rc in (0, 1), rc
    return B, (bad.value if rc else None)


def ref_echelon_zp(p, A, classical=False):
    A = _c(A, np.uint32).copy()
    m, n = A.shape
    r = _S(0); d = _U(0)
    fn = ref().lela_ref_elim_echelon_zp_u32 if classical else ref().lela_ref_echelon_zp_u32
    if fn(p, m, n, _ptr(A), n, ctypes.byref(r), ctypes.byref(d)):
        raise ArithmeticError("pivot not invertible")
    return A, r.value, d.value


def ref_echelon_reduced_zp(p, A, unit=False):
    """unit: Elimination::echelonize_reduced (the standard method)."""
    A = _c(A, np.uint32).copy()
    m, n = A.shape
    r = _S(0); d = _U(0)
    fn = ref().lela_ref_elim_echelon_reduced_zp_u32 if unit else ref().lela_ref_echelon_reduced_zp_u32
    if fn(p, m, n, _ptr(A), n, ctypes.byref(r), ctypes.byref(d)):
        raise ArithmeticError("pivot not invertible")
    return A, r.value, d.value


def ref_fl_echelonize_zp(p, m, n, rowptr, colidx, vals, reduced=True, only_D=False):
    rowptr = _c(rowptr, np.uint64); colidx = _c(colidx, np.uint32); vals = _c(vals, np.uint32)
    R = np.zeros((max(m, 1), n), dtype=np.uint32)
    rk = _S(0); det = _U(0); rows = _S(0)
    st = ref().lela_ref_fl_echelonize_zp_u32(p, m, n, _ptr(rowptr), _ptr(colidx), _ptr(vals),
                                             int(reduced), int(only_D), _ptr(R), n,
                                             ctypes.byref(rk), ctypes.byref(det), ctypes.byref(rows))
    return dict(status=st, R=R[:rows.value] if st == 0 else None, rank=rk.value, det=det.value)


def ref_gemm_gf2(A, B, C, k, n, a=1, b=1):
    A = _c(A, np.uint64); B = _c(B, np.uint64); C = _c(C, np.uint64).copy()
    m = A.shape[0]
    ref().lela_ref_gemm_gf2(m, n, k, a, _ptr(A), A.shape[1], _ptr(B), B.shape[1], b, _ptr(C), C.shape[1])
    return C


def ref_echelon_gf2(A, n):
    A = _c(A, np.uint64).copy()
    r = _S(0)
    ref().lela_ref_echelon_gf2(A.shape[0], n, _ptr(A), A.shape[1], ctypes.byref(r))
    return A, r.value


# ------------------------------------------------ LELA's matrix I/O (live)

def ref_detect_format(text):
    """MatrixReader::detectFormat (lela/matrix/io.tcc:163-200)."""
    return ref().lela_ref_detect_format(text.encode())


def ref_read_dumas(p, text, cap=1 << 22):
    """MatrixReader::read (FORMAT_DUMAS): (status, dense matrix or None);
    status 0 ok, 1 InvalidMatrixInput, 2 another exception."""
    m = _S(0); n = _S(0)
    A = np.zeros(cap, dtype=np.uint32)
    st = ref().lela_ref_read_dumas(p, text.encode(), cap, ctypes.byref(m), ctypes.byref(n), _ptr(A))
    if st:
        return st, None
    return 0, A[:m.value * n.value].reshape(m.value, n.value).copy()


def ref_write_dumas(p, A):
    """MatrixWriter::write (FORMAT_DUMAS) of a dense matrix."""
    A = _c(A, np.uint32)
    m, n = A.shape
    cap = 64 + 40 * int(np.count_nonzero(A)) + 64
    buf = ctypes.create_string_buffer(cap)
    ln = _S(0)
    st = ref().lela_ref_write_dumas(p, m, n, _ptr(A), max(n, 1), buf, cap, ctypes.byref(ln))
    assert st == 0
    return buf.value.decode()


def ref_write_matrix(fmt, p, A):
    """MatrixWriter::write (format fmt, a FileFormatTag) of a dense matrix."""
    A = _c(A, np.uint32)
    m, n = A.shape
    cap = 256 + 24 * m * max(n, 1)
    buf = ctypes.create_string_buffer(cap)
    ln = _S(0)
    st = ref().lela_ref_write_matrix(fmt, p, m, n, _ptr(A), max(n, 1), buf, cap, ctypes.byref(ln))
    assert st == 0
    return buf.value.decode()


def ref_read_matrix(fmt, p, text, m, n):
    """MatrixReader::read (format fmt) into an m x n matrix: (status, A)."""
    A = np.zeros((m, n), dtype=np.uint32)
    st = ref().lela_ref_read_matrix(fmt, p, text.encode(), m, n, _ptr(A))
    return st, (A if st == 0 else None)


def ref_pluq_zp(p, A):
    """Elimination::pluq (LELA): (LU in place, P, Q, rank, det)."""
    return _pluq(ref().lela_ref_pluq_zp_u32, p, A)


def ref_echelon_reduced_L_zp(p, A):
    """Elimination::echelonize_reduced with compute_L (LELA):
    (R, L, P, rank, det)."""
    return _echelon_L(ref().lela_ref_elim_echelon_reduced_L_zp_u32, p, A)


def ref_echelon_packed_L_zp(p, A, gauss_jordan=False):
    """Elimination::echelonize / GaussJordan::echelonize with L kept below
    the diagonal (LELA): (A, P, rank, det)."""
    return _packed(ref().lela_ref_echelon_packed_L_zp_u32, int(gauss_jordan), p, A)


def ref_gj_echelon_reduced_L_zp(p, A):
    """GaussJordan::echelonize_reduced with its transform (LELA):
    (R, L, P, rank, det)."""
    return _echelon_L(ref().lela_ref_gj_echelon_reduced_L_zp_u32, p, A)
