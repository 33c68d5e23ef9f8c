"""Host-side mirror of LELA's BLAS3 / algorithm interface for the CUDA module.

``CudaModule`` plays the role of a LELA ``Context<Ring, CUDAModule>``
(lela/blas/context.h:72-84): it owns one handle of the C ABI
(include/lela_cuda.h) -- a CUDA stream, device workspace and kernel choice.
Operation names and argument order follow LELA:

    gemm(p, a, A, B, b, C)          BLAS3::gemm     (lela/blas/level3.h:82)
    trsm(p, a, A, B, upper, unit)   BLAS3::trsm     (lela/blas/level3.h:121)

NumPy arrays are host matrices (uint32 for Z/p, uint64 words for GF(2));
torch CUDA tensors are device matrices and take the ``*_dev`` entry points.
Status codes become LELA's exceptions.
"""
import bisect
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))

_P = ctypes.c_void_p
_S = ctypes.c_size_t
_U = ctypes.c_uint32
_I = ctypes.c_int

OK, ERR_ARG, ERR_CUDA, ERR_NOMEM, DIAG, WRONG_FORM, PIVOT, TIMEOUT, UNSUPPORTED, ERR_CAPACITY = range(10)
GEMM_AUTO, GEMM_PLAIN, GEMM_TC, GEMM_SMALLK = 0, 1, 2, 3
GEMM_TILE_AUTO, GEMM_TILE_WIDE, GEMM_TILE_DOUBLE = 0, 1, 2
TRSM_AUTO, TRSM_BLOCKS, TRSM_INVERSE = 0, 1, 2


class LELAError(Exception):
    """LELAError (lela/util/error.h)."""


class PreconditionFailed(LELAError):
    """lela_check failure (lela/util/debug.h): bad dimensions or arguments."""


class DiagonalEntryNotInvertible(LELAError):
    """Thrown by trsm for a singular diagonal entry
    (lela/blas/level3-generic.tcc:441-442); ``idx`` is its row index."""

    def __init__(self, idx):
        super().__init__("Diagonal entry %d not invertible" % idx)
        self.idx = idx


class WrongMatrixForm(LELAError):
    """Bad Faugere-Lachartre input at ``row``
    (lela/algorithms/faugere-lachartre.tcc:32-41)."""

    def __init__(self, row):
        super().__init__("Bad input-matrix for Faugere-Lachartre at row-index %d" % row)
        self.row = row


class CudaError(LELAError):
    """CUDA runtime failure, device-side timeout or missing device."""


def library_path():
    return os.path.join(_HERE, "liblela_cuda.so")


_lib = None


def load_library():
    """Load liblela_cuda.so; raises (no fallback) when it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    path = library_path()
    if not os.path.exists(path):
        raise CudaError("CUDA library %s is not built (run python -m lela_b200.build)" % path)
    L = ctypes.CDLL(path)
    L.lela_cuda_create.argtypes = [ctypes.POINTER(_P), _I]
    L.lela_cuda_destroy.argtypes = [_P]
    L.lela_cuda_set_stream.argtypes = [_P, _P]
    L.lela_cuda_get_stream.argtypes = [_P]
    L.lela_cuda_get_stream.restype = _P
    L.lela_cuda_synchronize.argtypes = [_P]
    L.lela_cuda_set_gemm_kernel.argtypes = [_P, _I]
    L.lela_cuda_status_string.argtypes = [_I]
    L.lela_cuda_status_string.restype = ctypes.c_char_p
    L.lela_cuda_last_error.argtypes = [_P]
    L.lela_cuda_last_error.restype = ctypes.c_char_p
    L.lela_cuda_num_sms.argtypes = [_P]
    L.lela_cuda_launch_count.argtypes = [_P]
    L.lela_cuda_launch_count.restype = ctypes.c_uint64
    L.lela_cuda_profile_enable.argtypes = [_P, _I]
    L.lela_cuda_profile_read.argtypes = [_P, ctypes.c_char_p, ctypes.POINTER(ctypes.c_double),
                                         ctypes.POINTER(ctypes.c_uint64)]
    L.lela_cuda_profile_reset.argtypes = [_P]
    gemm_args = [_P, _S, _S, _S, _U, _U, _P, _S, _P, _S, _U, _P, _S]
    L.lela_cuda_gemm_zp_u32.argtypes = gemm_args
    L.lela_cuda_gemm_zp_u32_dev.argtypes = gemm_args
    _bind_optional(L)
    _lib = L
    return L


def _bind_optional(L):
    """Argument types of the entry points added alongside gemm."""
    sigs = {
        "lela_cuda_gemm_zp": [_P, _I, _S, _S, _S, _U, _U, _P, _S, _P, _S, _U, _P, _S],
        "lela_cuda_gemm_zp_dev": [_P, _I, _S, _S, _S, _U, _U, _P, _S, _P, _S, _U, _P, _S],
        "lela_cuda_trsm_zp": [_P, _I, _I, _I, _S, _S, _U, _U, _P, _S, _P, _S, ctypes.POINTER(_S)],
        "lela_cuda_trsm_zp_dev": [_P, _I, _I, _I, _S, _S, _U, _U, _P, _S, _P, _S, ctypes.POINTER(_S)],
        "lela_cuda_trsm_zp_u32": [_P, _I, _I, _S, _S, _U, _U, _P, _S, _P, _S, ctypes.POINTER(_S)],
        "lela_cuda_trsm_zp_u32_dev": [_P, _I, _I, _S, _S, _U, _U, _P, _S, _P, _S, ctypes.POINTER(_S)],
        "lela_cuda_trsm_csr_upper_zp_u32": [_P, _S, _S, _U, _U, _I, _P, _P, _P, _P, _S, ctypes.POINTER(_S)],
        "lela_cuda_trsm_csr_upper_zp_u32_dev": [_P, _S, _S, _U, _U, _I, _P, _P, _P, _P, _S, ctypes.POINTER(_S)],
        "lela_cuda_echelon_zp_u32": [_P, _S, _S, _U, _P, _S, ctypes.POINTER(_S), ctypes.POINTER(_U)],
        "lela_cuda_echelon_zp_u32_dev": [_P, _S, _S, _U, _P, _S, ctypes.POINTER(_S), ctypes.POINTER(_U)],
        "lela_cuda_echelon_reduced_zp_u32": [_P, _S, _S, _U, _P, _S, _I, ctypes.POINTER(_S),
                                             ctypes.POINTER(_U)],
        "lela_cuda_echelon_reduced_zp_u32_dev": [_P, _S, _S, _U, _P, _S, _I, ctypes.POINTER(_S),
                                                 ctypes.POINTER(_U)],
        "lela_cuda_fl_echelonize_zp_u32": [_P, _S, _S, _U, _P, _P, _P, _I, _I, _P, _S,
                                           ctypes.POINTER(_S), ctypes.POINTER(_U),
                                           ctypes.POINTER(_S), ctypes.POINTER(_S)],
        "lela_cuda_fl_echelonize_zp_u32_dev": [_P, _S, _S, _U, _P, _P, _P, _I, _I, _P, _S,
                                               ctypes.POINTER(_S), ctypes.POINTER(_U),
                                               ctypes.POINTER(_S), ctypes.POINTER(_S)],
        "lela_cuda_fl_echelonize_zp_u32_csr": [_P, _S, _S, _U, _P, _P, _P, _I, _I, _P, _P, _P, _S,
                                               ctypes.POINTER(_S), ctypes.POINTER(_S),
                                               ctypes.POINTER(_U), ctypes.POINTER(_S),
                                               ctypes.POINTER(_S)],
        "lela_cuda_fl_echelonize_zp_u32_csr_dev": [_P, _S, _S, _U, _P, _P, _P, _I, _I, _P, _P, _P, _S,
                                                   ctypes.POINTER(_S), ctypes.POINTER(_S),
                                                   ctypes.POINTER(_U), ctypes.POINTER(_S),
                                                   ctypes.POINTER(_S)],
        "lela_cuda_fl_csr_fetch": [_P, _P, _P, _S, _I],
        "lela_cuda_pluq_zp_u32": [_P, _S, _S, _U, _P, _S, _P, ctypes.POINTER(_S), _P,
                                  ctypes.POINTER(_S), ctypes.POINTER(_S), ctypes.POINTER(_U)],
        "lela_cuda_pluq_zp_u32_dev": [_P, _S, _S, _U, _P, _S, _P, ctypes.POINTER(_S), _P,
                                      ctypes.POINTER(_S), ctypes.POINTER(_S), ctypes.POINTER(_U)],
        "lela_cuda_echelon_reduced_transform_zp_u32": [_P, _S, _S, _U, _P, _S, _P, _S, _P,
                                                       ctypes.POINTER(_S), ctypes.POINTER(_S),
                                                       ctypes.POINTER(_U)],
        "lela_cuda_echelon_reduced_transform_zp_u32_dev": [_P, _S, _S, _U, _P, _S, _P, _S, _P,
                                                           ctypes.POINTER(_S), ctypes.POINTER(_S),
                                                           ctypes.POINTER(_U)],
        "lela_cuda_gemm_gf2": [_P, _S, _S, _S, _I, _P, _S, _P, _S, _I, _P, _S],
        "lela_cuda_gemm_gf2_dev": [_P, _S, _S, _S, _I, _P, _S, _P, _S, _I, _P, _S],
        "lela_cuda_echelon_gf2": [_P, _S, _S, _P, _S, ctypes.POINTER(_S)],
        "lela_cuda_echelon_gf2_dev": [_P, _S, _S, _P, _S, ctypes.POINTER(_S)],
        "lela_cuda_set_gf2_kernel": [_P, _I],
        "lela_cuda_set_gemm_tile": [_P, _I],
        "lela_cuda_set_trsm_kernel": [_P, _I],
        "lela_cuda_set_batch_memory_budget": [_P, _S],
    }
    for name, args in sigs.items():
        if hasattr(L, name):
            getattr(L, name).argtypes = args


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _dptr(t):
    return ctypes.c_void_p(t.data_ptr())


# Element types of Modular<T> (include/lela_cuda.h, enum lela_cuda_elem).
ELEM_U8, ELEM_U16, ELEM_U32, ELEM_F32, ELEM_F64 = 1, 2, 4, 5, 6


def _elem_of(X):
    """(element code, bytes per element) of a numpy array or torch tensor:
    uint8, uint16 (torch int16 / uint16), uint32 (torch int32), float32,
    float64 -- the element types of Modular<uint8/uint16/uint32/float/double>."""
    if _is_torch(X):
        import torch
        table = {torch.uint8: ELEM_U8, torch.int16: ELEM_U16, torch.int32: ELEM_U32,
                 torch.float32: ELEM_F32, torch.float64: ELEM_F64}
        if hasattr(torch, "uint16"):
            table[torch.uint16] = ELEM_U16
        if hasattr(torch, "uint32"):
            table[torch.uint32] = ELEM_U32
        code = table.get(X.dtype)
        _check(code is not None, "unsupported element type %s" % X.dtype)
        return code, X.element_size()
    table = {np.dtype(np.uint8): ELEM_U8, np.dtype(np.uint16): ELEM_U16,
             np.dtype(np.uint32): ELEM_U32, np.dtype(np.float32): ELEM_F32,
             np.dtype(np.float64): ELEM_F64}
    code = table.get(X.dtype)
    _check(code is not None, "unsupported element type %s" % X.dtype)
    return code, X.itemsize


class CudaModule:
    """One handle of the CUDA module on ``device`` (default 0)."""

    def __init__(self, device=0):
        self.L = load_library()
        h = _P()
        st = self.L.lela_cuda_create(ctypes.byref(h), int(device))
        if st != OK:
            raise CudaError("lela_cuda_create(device=%d) failed: %s" %
                            (device, self.L.lela_cuda_status_string(st).decode()))
        self.h = h
        self.device = device

    def close(self):
        if getattr(self, "h", None):
            self.L.lela_cuda_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---------------------------------------------------------------- misc
    def _raise(self, st, aux=0):
        if st == OK:
            return
        msg = self.L.lela_cuda_last_error(self.h).decode()
        if st == DIAG:
            raise DiagonalEntryNotInvertible(aux)
        if st == WRONG_FORM:
            raise WrongMatrixForm(aux)
        if st == PIVOT:
            raise LELAError("Could not invert pivot-element in the ring")
        if st == ERR_ARG:
            raise PreconditionFailed(msg)
        raise CudaError("%s: %s" % (self.L.lela_cuda_status_string(st).decode(), msg))

    def set_stream(self, stream):
        """Run on a caller stream (cudaStream_t as int / torch.cuda.Stream)."""
        handle = getattr(stream, "cuda_stream", stream)
        self._raise(self.L.lela_cuda_set_stream(self.h, _P(handle)))

    def stream(self):
        return self.L.lela_cuda_get_stream(self.h)

    def synchronize(self):
        self._raise(self.L.lela_cuda_synchronize(self.h))

    def set_gemm_kernel(self, kernel):
        self._raise(self.L.lela_cuda_set_gemm_kernel(self.h, int(kernel)))

    def set_gemm_tile(self, tile):
        """Tensor-core tile variant: 0 = automatic, 1 = wide tiles (one
        accumulator buffer), 2 = narrower tiles with two accumulator buffers
        (one and two limbs).  Results do not depend on it."""
        self._raise(self.L.lela_cuda_set_gemm_tile(self.h, int(tile)))

    @property
    def num_sms(self):
        return self.L.lela_cuda_num_sms(self.h)

    @property
    def launch_count(self):
        """Kernel launches issued through this handle so far."""
        return int(self.L.lela_cuda_launch_count(self.h))

    def profile(self, on=True):
        self._raise(self.L.lela_cuda_profile_enable(self.h, int(on)))

    def profile_read(self, kernel):
        """(total device ms, launches) of one kernel since the last read."""
        ms = ctypes.c_double(0)
        n = ctypes.c_uint64(0)
        self._raise(self.L.lela_cuda_profile_read(self.h, kernel.encode(), ctypes.byref(ms),
                                                  ctypes.byref(n)))
        return ms.value, int(n.value)

    def profile_reset(self):
        self._raise(self.L.lela_cuda_profile_reset(self.h))

    # ---------------------------------------------------------- Z/p gemm
    def gemm(self, p, a, A, B, b, C):
        """C <- a*A*B + b*C mod p in place (BLAS3::gemm); returns C.
        Host numpy matrices or torch CUDA tensors of one element type:
        uint32 (torch int32), or the element types of Modular<uint8>,
        Modular<uint16>, Modular<float>, Modular<double> (uint8, uint16,
        float32, float64; float entries are the symmetric representatives
        -p/2 .. p/2)."""
        elem, es = _elem_of(C)
        if elem != ELEM_U32:
            _check(_elem_of(A)[0] == elem and _elem_of(B)[0] == elem, "gemm: mixed element types")
            m, n = C.shape
            k = A.shape[1]
            _check(A.shape[0] == m and B.shape == (k, n), "gemm: dimension mismatch")
            if _is_torch(C):
                st = self.L.lela_cuda_gemm_zp_dev(self.h, elem, m, n, k, p, a % p, _dptr(A),
                                                  A.stride(0), _dptr(B), B.stride(0), b % p,
                                                  _dptr(C), C.stride(0))
            else:
                _check(C.flags.c_contiguous or C.strides[1] == es, "gemm: rows of C must be contiguous")
                A = np.ascontiguousarray(A)
                B = np.ascontiguousarray(B)
                st = self.L.lela_cuda_gemm_zp(self.h, elem, m, n, k, p, a % p, _ptr(A), A.strides[0] // es,
                                              _ptr(B), B.strides[0] // es, b % p, _ptr(C),
                                              C.strides[0] // es)
            self._raise(st)
            return C
        if _is_torch(C):
            m, n = C.shape
            k = A.shape[1]
            _check(A.shape[0] == m and B.shape == (k, n), "gemm: dimension mismatch")
            st = self.L.lela_cuda_gemm_zp_u32_dev(self.h, m, n, k, p, a % p, _dptr(A), A.stride(0),
                                                  _dptr(B), B.stride(0), b % p, _dptr(C), C.stride(0))
            self._raise(st)
            return C
        _check(C.dtype == np.uint32 and A.dtype == np.uint32 and B.dtype == np.uint32,
               "gemm: uint32 matrices expected")
        m, n = C.shape
        k = A.shape[1]
        _check(A.shape[0] == m and B.shape == (k, n), "gemm: dimension mismatch")
        _check(C.flags.c_contiguous or C.strides[1] == 4, "gemm: rows of C must be contiguous")
        st = self.L.lela_cuda_gemm_zp_u32(self.h, m, n, k, p, a % p, _ptr(A), A.strides[0] // 4,
                                          _ptr(B), B.strides[0] // 4, b % p, _ptr(C), C.strides[0] // 4)
        self._raise(st)
        return C


    # ---------------------------------------------------------- Z/p trsm
    def trsm(self, p, a, A, B, upper, diag_is_one=False):
        """B <- a*A^-1*B mod p in place (BLAS3::trsm with UpperTriangular /
        LowerTriangular); raises DiagonalEntryNotInvertible(idx)."""
        m = A.shape[0]
        _check(A.shape == (m, m) and B.shape[0] == m, "trsm: dimension mismatch")
        n = B.shape[1]
        bad = _S(0)
        elem, es = _elem_of(B)
        if elem != ELEM_U32:
            _check(_elem_of(A)[0] == elem, "trsm: mixed element types")
            if _is_torch(B):
                st = self.L.lela_cuda_trsm_zp_dev(self.h, elem, int(upper), int(diag_is_one), m, n, p,
                                                  a % p, _dptr(A), A.stride(0), _dptr(B), B.stride(0),
                                                  ctypes.byref(bad))
            else:
                _check(B.flags.c_contiguous or B.strides[1] == es, "trsm: rows of B must be contiguous")
                A = np.ascontiguousarray(A)
                st = self.L.lela_cuda_trsm_zp(self.h, elem, int(upper), int(diag_is_one), m, n, p,
                                              a % p, _ptr(A), A.strides[0] // es, _ptr(B),
                                              B.strides[0] // es, ctypes.byref(bad))
            self._raise(st, bad.value)
            return B
        if _is_torch(B):
            st = self.L.lela_cuda_trsm_zp_u32_dev(self.h, int(upper), int(diag_is_one), m, n, p,
                                                  a % p, _dptr(A), A.stride(0), _dptr(B), B.stride(0),
                                                  ctypes.byref(bad))
        else:
            _check(A.dtype == np.uint32 and B.dtype == np.uint32, "trsm: uint32 matrices expected")
            st = self.L.lela_cuda_trsm_zp_u32(self.h, int(upper), int(diag_is_one), m, n, p, a % p,
                                              _ptr(A), A.strides[0] // 4, _ptr(B), B.strides[0] // 4,
                                              ctypes.byref(bad))
        self._raise(st, bad.value)
        return B

    def trsm_csr_upper(self, p, a, n, rowptr, colidx, vals, B, diag_is_one=False):
        """B <- a*A^-1*B mod p in place for an n x n upper-triangular A in CSR
        form (BLAS3::trsm on a SparseMatrix, as in FaugereLachartre's A^-1 B);
        numpy arrays (host) or torch CUDA tensors (device: rowptr int64,
        colidx / vals int32, B int32).  Raises DiagonalEntryNotInvertible(idx)."""
        _check(B.shape[0] == n and len(rowptr) == n + 1, "trsm_csr_upper: dimension mismatch")
        ncols = B.shape[1]
        bad = _S(0)
        if _is_torch(B):
            st = self.L.lela_cuda_trsm_csr_upper_zp_u32_dev(
                self.h, n, ncols, p, a % p, int(diag_is_one), _dptr(rowptr), _dptr(colidx),
                _dptr(vals), _dptr(B), B.stride(0), ctypes.byref(bad))
        else:
            _check(B.dtype == np.uint32 and rowptr.dtype == np.uint64 and colidx.dtype == np.uint32
                   and vals.dtype == np.uint32, "trsm_csr_upper: uint64 rowptr, uint32 colidx/vals/B")
            st = self.L.lela_cuda_trsm_csr_upper_zp_u32(
                self.h, n, ncols, p, a % p, int(diag_is_one), _ptr(rowptr), _ptr(colidx),
                _ptr(vals), _ptr(B), B.strides[0] // 4, ctypes.byref(bad))
        self._raise(st, bad.value)
        return B


    # ------------------------------------------------------- echelon form
    def echelonize(self, p, A, reduced=False, unit_pivots=False):
        """A <- row-echelon form in place (EchelonForm::echelonize (A,
        reduced) on a DenseMatrix, LELA's pivot rule; reduced: zero above and
        below the pivots, which keep their values, or with unit_pivots are
        divided out as the standard method does); returns (A, rank, det)."""
        m, n = A.shape
        r = _S(0)
        d = _U(0)
        name = "lela_cuda_echelon_reduced_zp_u32" if reduced else "lela_cuda_echelon_zp_u32"
        extra = (int(bool(unit_pivots)),) if reduced else ()
        if _is_torch(A):
            st = getattr(self.L, name + "_dev")(self.h, m, n, p, _dptr(A), A.stride(0), *extra,
                                                ctypes.byref(r), ctypes.byref(d))
        else:
            _check(A.dtype == np.uint32, "echelonize: uint32 matrix expected")
            st = getattr(self.L, name)(self.h, m, n, p, _ptr(A), A.strides[0] // 4, *extra,
                                       ctypes.byref(r), ctypes.byref(d))
        self._raise(st)
        return A, r.value, d.value


    def echelonize_with_L(self, p, A, gauss_jordan=False):
        """Elimination::echelonize (A, P, rank, det) with its default
        compute_L = true (lela/algorithms/elimination.h:86-92,
        elimination.tcc:47-139), or with gauss_jordan GaussJordan::
        echelonize (A, P, rank, det) (gauss-jordan.tcc:413-432), in place:
        A <- the non-reduced form U with, below the diagonal, the strictly
        lower part of the unit lower triangular T with T P A_in = U; returns
        (A, P, rank, det), P the transpositions in the order applied.  Both
        give the same A and P; det is the product of the pivots for
        Elimination and GaussTransform's d for GaussJordan
        (gauss_transform_det).

        In blocks of rank rows T = [[L1^-1, 0], [-L2 L1^-1, I]] (B = P A =
        [L1; L2] U), so its bottom block is that of the reduced form's
        transform and its top block is U_P X, X the reduced transform's top
        block (X = U_P^-1 L1^-1, U_P the pivot columns of U).  Computed from
        the GPU's reduced transform, its non-reduced form and one gemm.
        Host arrays only; p < 2^31."""
        _check(not _is_torch(A), "echelonize_with_L takes host arrays")
        _check(A.dtype == np.uint32, "echelonize_with_L: uint32 matrix expected")
        m, n = A.shape
        _, T, P, r, d = self.echelon_reduced_transform(p, np.array(A, dtype=np.uint32, copy=True))
        if r == 0:
            return A, P, r, (1 % p if gauss_jordan else d)
        self.echelonize(p, A)
        piv = [int(np.flatnonzero(A[i])[0]) for i in range(r)]
        vals = [int(A[i, c]) for i, c in enumerate(piv)]
        UP = np.ascontiguousarray(A[:r][:, piv])
        X = np.ascontiguousarray(T[:r, :r])
        T11 = self.gemm(p, 1, UP, X, 0, np.zeros((r, r), dtype=np.uint32))
        for i in range(1, r):
            A[i, :i] = T11[i, :i]
        A[r:, :r] = T[r:, :r]
        if gauss_jordan:
            d = gauss_transform_det(p, n, piv, vals)
        return A, P, r, d

    def pluq(self, p, A):
        """Elimination::pluq in place: A <- L below the diagonal and U on and
        above it (columns in Q's order); returns (A, P, Q, rank, det) with P
        and Q lists of transposition pairs in the reference's order.  Host
        numpy uint32 matrix or torch CUDA tensor."""
        m, n = A.shape
        k = max(min(m, n), 1)
        P = np.zeros(2 * k, dtype=np.uint64)
        Q = np.zeros(2 * k, dtype=np.uint64)
        np_, nq, r, d = _S(0), _S(0), _S(0), _U(0)
        if _is_torch(A):
            st = self.L.lela_cuda_pluq_zp_u32_dev(self.h, m, n, p, _dptr(A), A.stride(0), _ptr(P),
                                                  ctypes.byref(np_), _ptr(Q), ctypes.byref(nq),
                                                  ctypes.byref(r), ctypes.byref(d))
        else:
            _check(A.dtype == np.uint32, "pluq: uint32 matrix expected")
            st = self.L.lela_cuda_pluq_zp_u32(self.h, m, n, p, _ptr(A), A.strides[0] // 4, _ptr(P),
                                              ctypes.byref(np_), _ptr(Q), ctypes.byref(nq),
                                              ctypes.byref(r), ctypes.byref(d))
        self._raise(st)
        pairs = lambda X, c: [(int(X[2 * t]), int(X[2 * t + 1])) for t in range(c)]
        return A, pairs(P, np_.value), pairs(Q, nq.value), r.value, d.value

    def echelon_reduced_transform(self, p, A, L=None, unit_pivots=True):
        """Elimination::echelonize_reduced (A, L, P, rank, det, compute_L =
        true): A <- its reduced form with unit pivots, in place; returns (A,
        L, P, rank, det) with A_out = L P A_in, L m x m, and P a list of
        transposition pairs in the order applied.  Host numpy uint32 matrix,
        or torch CUDA tensor (then L is a device tensor too).  p < 2^31.

        unit_pivots=False: GaussJordan::echelonize_reduced (A, L, P, rank,
        det) instead (lela/algorithms/gauss-jordan.tcc:434-466), whose
        pivots keep their values.  Its transposition list is the standard
        method's, and its pivot rows of A and L are the standard method's
        multiplied by their pivots (GaussJordanTransform's leaf leaves the
        pivot row as it is, :74-107).  So it is the standard form, with the
        pivots read from the fast method's reduced form
        (lela_cuda_echelon_reduced_zp_u32 with unit_pivots = 0) of the same
        input.  Host arrays only."""
        if not unit_pivots:
            _check(not _is_torch(A), "echelon_reduced_transform: the fast method's form takes host arrays")
            A0 = np.array(A, dtype=np.uint32, copy=True)
            A, L, P, r, d = self.echelon_reduced_transform(p, A, L)
            if r:
                Rg, _, _ = self.echelonize(p, A0, reduced=True, unit_pivots=False)
                A[:r] = Rg[:r]
                scale_pivot_rows(p, L, Rg, r)
            return A, L, P, r, d
        m, n = A.shape
        P = np.zeros(2 * max(min(m, n), 1), dtype=np.uint64)
        np_, r, d = _S(0), _S(0), _U(0)
        if _is_torch(A):
            import torch
            if L is None:
                L = torch.empty((m, m), dtype=A.dtype, device=A.device)
            st = self.L.lela_cuda_echelon_reduced_transform_zp_u32_dev(
                self.h, m, n, p, _dptr(A), max(A.stride(0), 1), _dptr(L), max(L.stride(0), 1),
                _ptr(P), ctypes.byref(np_), ctypes.byref(r), ctypes.byref(d))
        else:
            _check(A.dtype == np.uint32, "echelon_reduced_transform: uint32 matrix expected")
            if L is None:
                L = np.zeros((m, m), dtype=np.uint32)
            st = self.L.lela_cuda_echelon_reduced_transform_zp_u32(
                self.h, m, n, p, _ptr(A), max(A.strides[0] // 4, n, 1), _ptr(L),
                max(L.strides[0] // 4, m, 1), _ptr(P), ctypes.byref(np_), ctypes.byref(r),
                ctypes.byref(d))
        self._raise(st)
        return A, L, [(int(P[2 * t]), int(P[2 * t + 1])) for t in range(np_.value)], r.value, d.value

    # ------------------------------------------------- Faugere-Lachartre
    def fl_echelonize(self, p, X, reduced=True, only_D=False, R=None):
        """FaugereLachartre::echelonize of the CSR matrix X (an object with
        m, n, rowptr, colidx, vals -- numpy arrays for the host path, torch
        CUDA tensors for the device path).  Returns (R, rank, det); R is the
        dense output (out_rows x n).  Raises WrongMatrixForm(row); a singular
        pivot block raises DiagonalEntryNotInvertible (the reference returns
        early there)."""
        m, n = X.m, X.n
        rk, det, rows, bad = _S(0), _U(0), _S(0), _S(0)
        if _is_torch(X.rowptr):
            import torch
            if R is None:
                R = torch.empty((max(m, 1), n), dtype=torch.int32, device=X.rowptr.device)
            st = self.L.lela_cuda_fl_echelonize_zp_u32_dev(
                self.h, m, n, p, _dptr(X.rowptr), _dptr(X.colidx), _dptr(X.vals), int(reduced),
                int(only_D), _dptr(R), R.stride(0), ctypes.byref(rk), ctypes.byref(det),
                ctypes.byref(rows), ctypes.byref(bad))
        else:
            if R is None:
                R = np.zeros((max(m, 1), n), dtype=np.uint32)
            rowptr = np.ascontiguousarray(X.rowptr, dtype=np.uint64)
            colidx = np.ascontiguousarray(X.colidx, dtype=np.uint32)
            vals = np.ascontiguousarray(X.vals, dtype=np.uint32)
            st = self.L.lela_cuda_fl_echelonize_zp_u32(
                self.h, m, n, p, _ptr(rowptr), _ptr(colidx), _ptr(vals), int(reduced), int(only_D),
                _ptr(R), R.strides[0] // 4, ctypes.byref(rk), ctypes.byref(det), ctypes.byref(rows),
                ctypes.byref(bad))
        self._raise(st, bad.value)
        return R[:rows.value], rk.value, det.value


    def fl_echelonize_csr(self, p, X, reduced=True, only_D=False, cap=None):
        """FaugereLachartre::echelonize with the result as CSR rows (the
        SparseMatrix the reference writes; no dense m x n array).  X as for
        fl_echelonize (numpy arrays: host path; torch CUDA tensors: device
        path, output tensors on the device).  Returns (R, rank, det) with R
        a gen.CSR of out_rows rows (host) or an object with m, n, rowptr,
        colidx, vals tensors (device).  cap: first guess of the entry count
        (the result is fetched again when it holds more)."""
        m, n = X.m, X.n
        rk, det, rows, bad, nnz = _S(0), _U(0), _S(0), _S(0), _S(0)
        if _is_torch(X.rowptr):
            import torch
            import types
            dev = X.rowptr.device
            cap = int(cap if cap is not None else max(1, 2 * int(X.colidx.numel())))
            rp = torch.empty(m + 1, dtype=torch.int64, device=dev)
            ci = torch.empty(max(cap, 1), dtype=torch.int32, device=dev)
            va = torch.empty(max(cap, 1), dtype=torch.int32, device=dev)
            st = self.L.lela_cuda_fl_echelonize_zp_u32_csr_dev(
                self.h, m, n, p, _dptr(X.rowptr), _dptr(X.colidx), _dptr(X.vals), int(reduced),
                int(only_D), _dptr(rp), _dptr(ci), _dptr(va), cap, ctypes.byref(nnz),
                ctypes.byref(rk), ctypes.byref(det), ctypes.byref(rows), ctypes.byref(bad))
            if st == ERR_CAPACITY:
                ci = torch.empty(max(nnz.value, 1), dtype=torch.int32, device=dev)
                va = torch.empty(max(nnz.value, 1), dtype=torch.int32, device=dev)
                st = self.L.lela_cuda_fl_csr_fetch(self.h, _dptr(ci), _dptr(va), nnz.value, 1)
            self._raise(st, bad.value)
            R = types.SimpleNamespace(m=rows.value, n=n, rowptr=rp[:rows.value + 1],
                                      colidx=ci[:nnz.value], vals=va[:nnz.value])
            return R, rk.value, det.value
        rowptr = np.ascontiguousarray(X.rowptr, dtype=np.uint64)
        colidx = np.ascontiguousarray(X.colidx, dtype=np.uint32)
        vals = np.ascontiguousarray(X.vals, dtype=np.uint32)
        cap = int(cap if cap is not None else max(1, 2 * len(colidx)))
        rp = np.zeros(m + 1, dtype=np.uint64)
        ci = np.zeros(max(cap, 1), dtype=np.uint32)
        va = np.zeros(max(cap, 1), dtype=np.uint32)
        st = self.L.lela_cuda_fl_echelonize_zp_u32_csr(
            self.h, m, n, p, _ptr(rowptr), _ptr(colidx), _ptr(vals), int(reduced), int(only_D),
            _ptr(rp), _ptr(ci), _ptr(va), cap, ctypes.byref(nnz), ctypes.byref(rk),
            ctypes.byref(det), ctypes.byref(rows), ctypes.byref(bad))
        if st == ERR_CAPACITY:
            ci = np.zeros(max(nnz.value, 1), dtype=np.uint32)
            va = np.zeros(max(nnz.value, 1), dtype=np.uint32)
            st = self.L.lela_cuda_fl_csr_fetch(self.h, _ptr(ci), _ptr(va), nnz.value, 0)
        self._raise(st, bad.value)
        from .gen import CSR
        return (CSR(rows.value, n, rp[:rows.value + 1], ci[:nnz.value], va[:nnz.value]),
                rk.value, det.value)

    # ------------------------------------------------------------- GF(2)
    def set_gf2_kernel(self, kernel):
        """0 = auto (tensor cores), 1 = int8-expanded tcgen05, 2 = M4RM."""
        self._raise(self.L.lela_cuda_set_gf2_kernel(self.h, int(kernel)))

    def set_trsm_kernel(self, kernel):
        """0 = auto, 1 = 256-row block substitution, 2 = 512-row inverses on the tensor cores."""
        self._raise(self.L.lela_cuda_set_trsm_kernel(self.h, int(kernel)))

    def gemm_gf2(self, A, B, C, n, k, a=1, b=1):
        """C <- a*A*B + b*C over GF(2) in place; packed uint64 rows (bit j of
        word w = column 64w + j); n, k = bit widths of C/B and A."""
        m = C.shape[0]
        if _is_torch(C):
            st = self.L.lela_cuda_gemm_gf2_dev(self.h, m, n, k, int(a), _dptr(A), A.stride(0),
                                               _dptr(B), B.stride(0), int(b), _dptr(C), C.stride(0))
        else:
            _check(C.dtype == np.uint64 and A.dtype == np.uint64 and B.dtype == np.uint64,
                   "gemm_gf2: uint64 words expected")
            st = self.L.lela_cuda_gemm_gf2(self.h, m, n, k, int(a), _ptr(A), A.strides[0] // 8,
                                           _ptr(B), B.strides[0] // 8, int(b), _ptr(C),
                                           C.strides[0] // 8)
        self._raise(st)
        return C

    def echelonize_gf2(self, A, n):
        """A <- non-reduced row-echelon form over GF(2) in place; returns
        (A, rank)."""
        m = A.shape[0]
        r = _S(0)
        if _is_torch(A):
            st = self.L.lela_cuda_echelon_gf2_dev(self.h, m, n, _dptr(A), A.stride(0), ctypes.byref(r))
        else:
            _check(A.dtype == np.uint64, "echelonize_gf2: uint64 words expected")
            st = self.L.lela_cuda_echelon_gf2(self.h, m, n, _ptr(A), A.strides[0] // 8, ctypes.byref(r))
        self._raise(st)
        return A, r.value


    # ------------------------------------------------------------- batches
    def echelonize_batch(self, mats, ps, kernels=None):
        """Echelon forms of many dense device blocks (torch CUDA tensors,
        int32 storage) in place; ps = moduli; kernels per block as for
        lela_cuda_echelon_zp_u32_batch (0 auto, 1 shared-memory batch kernel,
        2 panels + tensor-core updates, 3 panels + CUDA-core updates).
        Returns (ranks, dets, statuses)."""
        n = len(mats)
        P = (ctypes.c_void_p * n)(*[t.data_ptr() for t in mats])
        lda = (_S * n)(*[t.stride(0) for t in mats])
        ms = (_S * n)(*[t.shape[0] for t in mats])
        ns = (_S * n)(*[t.shape[1] for t in mats])
        pp = (_U * n)(*ps)
        kk = (ctypes.c_int * n)(*(kernels or [0] * n))
        rk = (_S * n)()
        dt = (_U * n)()
        stt = (ctypes.c_int * n)()
        fn = self.L.lela_cuda_echelon_zp_u32_batch
        fn.argtypes = [_P, _S, _P, _P, _P, _P, _P, _P, _P, _P, _P]
        st = fn(self.h, n, ctypes.cast(P, _P), ctypes.cast(lda, _P), ctypes.cast(ms, _P),
                ctypes.cast(ns, _P), ctypes.cast(pp, _P), ctypes.cast(kk, _P), ctypes.cast(rk, _P),
                ctypes.cast(dt, _P), ctypes.cast(stt, _P))
        self._raise(st)
        return list(rk), list(dt), list(stt)

    def set_batch_memory_budget(self, nbytes):
        """Device-memory budget of fl_echelonize_batch (0 = automatic)."""
        self._raise(self.L.lela_cuda_set_batch_memory_budget(self.h, int(nbytes)))

    def fl_echelonize_batch(self, Xs, ps, Rs, reduced=True, nworkers=4):
        """Faugere-Lachartre on many device CSR matrices (objects with m, n,
        rowptr, colidx, vals as torch CUDA tensors) into device outputs Rs;
        returns (ranks, dets, statuses)."""
        n = len(Xs)
        arr = lambda vals, T: (T * n)(*vals)
        ptrs = lambda ts: (ctypes.c_void_p * n)(*[t.data_ptr() for t in ts])
        rk, dt, stt = (_S * n)(), (_U * n)(), (ctypes.c_int * n)()
        fn = self.L.lela_cuda_fl_echelonize_zp_u32_batch
        fn.argtypes = [_P, _S, _P, _P, _P, _P, _P, _P, _P, _P, _I, _I, _P, _P, _P]
        c = lambda x: ctypes.cast(x, _P)
        st = fn(self.h, n, c(arr([X.m for X in Xs], _S)), c(arr([X.n for X in Xs], _S)),
                c(arr(ps, _U)), c(ptrs([X.rowptr for X in Xs])), c(ptrs([X.colidx for X in Xs])),
                c(ptrs([X.vals for X in Xs])), c(ptrs(Rs)), c(arr([R.stride(0) for R in Rs], _S)),
                int(reduced), int(nworkers), c(rk), c(dt), c(stt))
        self._raise(st)
        return list(rk), list(dt), list(stt)


def _is_torch(x):
    return type(x).__module__.startswith("torch")


def gauss_transform_det(p, n, pivot_cols, pivot_vals):
    """The determinant GaussJordan::echelonize returns (lela/algorithms/
    gauss-jordan.tcc:232-411, GaussTransform's d), from the pivot columns
    (increasing) and pivot values of the non-reduced form.  The recursion
    halves the columns; a block without a pivot is zero and copies d_0 into
    d, a one-column block multiplies d by its pivot, and a wider block runs
    its left half with d_0 into d_1 = 1 and its right half with d_1 as d_0
    into d.  The top call has d_0 = d = 1."""
    cols = list(pivot_cols)
    val = dict(zip(cols, pivot_vals))

    def has(c0, c1):
        i = bisect.bisect_left(cols, c0)
        return i < len(cols) and cols[i] < c1

    def rec(c0, c1, d0, d):
        if not has(c0, c1):
            return d0
        if c1 - c0 == 1:
            return d * val[c0] % p
        m1 = (c1 - c0) // 2
        return rec(c0 + m1, c1, rec(c0, c0 + m1, d0, 1 % p), d)

    return rec(0, n, 1 % p, 1 % p) if n else 1 % p


def scale_pivot_rows(p, L, R, r):
    """L[i] <- x_i L[i] mod p for i < r, in place, x_i the leading entry of
    row i of R (a reduced echelon form whose first r rows are its pivot
    rows)."""
    for i in range(r):
        nz = np.flatnonzero(R[i])
        x = np.uint64(R[i, nz[0]])
        L[i] = (L[i].astype(np.uint64) * x % np.uint64(p)).astype(np.uint32)


def _check(cond, msg):
    if not cond:
        raise PreconditionFailed(msg)
