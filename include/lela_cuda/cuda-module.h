/* include/lela_cuda/cuda-module.h -- the CUDA module for LELA's compile-time
 * Context/Module dispatch.
 *
 * With
 *
 *     Modular<uint32> F (65521);
 *     Context<Modular<uint32>, CUDAModule<uint32> > ctx (F);
 *
 * BLAS3::gemm (ctx, a, A, B, b, C) and BLAS3::trsm (ctx, a, A, B, type,
 * diagIsOne) on DenseMatrix<uint32> operands run on the GPU through the C
 * ABI of include/lela_cuda.h, and FaugereLachartre<Modular<uint32>,
 * CUDAModule<uint32> >::echelonize runs the whole Faugere-Lachartre pipeline
 * there, as does EchelonForm<Modular<uint32>, CUDAModule<uint32> >::echelonize
 * for the dense echelon forms, reduced or not; BLAS3::trsm also takes a
 * sparse upper-triangular SparseMatrix<uint32> A.  With Context<Modular<T>,
 * CUDAModule<T> > for T = uint8, uint16, float or double, BLAS3::gemm and
 * BLAS3::trsm on DenseMatrix<T> operands run on the GPU.  With Context<GF2, CUDAModuleGF2>, BLAS3::gemm on DenseMatrix<bool>
 * operands runs on the GPU.  Operand combinations the GPU path does not take
 * (sparse gemm operands, sparse lower-triangular or transposed operands) fall
 * through to the parent module, exactly as an unimplemented operation falls
 * through LELA's module stack (lela/blas/context.h:109-146).
 *
 * Mechanism (the reference's own): a Modules class with a Tag whose Parent
 * is the next module (ZpModule<uint32>, lela/ring/modular.h:604-626), and
 * partial specialisations _gemm<Modular<uint32>, CUDAModule<uint32>::Tag>
 * and _trsm<...> of the class templates in lela/blas/level3-ll.h:52-75,
 * dispatched on MatrixStorageTypes as lela/blas/level3-modular.h:28-47 does.
 * Errors become LELA's exceptions: DiagonalEntryNotInvertible(idx)
 * (lela/util/error.h:83-91), WrongMatrixForm(row), LELAError.
 *
 * Header-only; include it after the LELA headers it names and link
 * liblela_cuda.so.  Written to compile as C++98 like LELA itself.
 */
#ifndef LELA_CUDA_CUDA_MODULE_H
#define LELA_CUDA_CUDA_MODULE_H

#include <cstdlib>
#include <map>
#include <vector>

#include "lela/blas/context.h"
#include "lela/blas/level3-ll.h"
#include "lela/matrix/dense.h"
#include "lela/matrix/sparse.h"
#include "lela/ring/modular.h"
#include "lela/ring/gf2.h"
#include "lela/util/error.h"
#include "lela/algorithms/faugere-lachartre.h"
#include "lela/algorithms/elimination.h"
#include "lela/algorithms/gauss-jordan.h"
#include "lela/solutions/echelon-form.h"

#include "../lela_cuda.h"

namespace LELA
{

/** Shared, reference-counted handle of the C ABI (one CUDA stream and
 * device workspace).  The device is taken from LELA_CUDA_DEVICE (default
 * 0).  A Context is not re-entrant (lela/blas/context.h:61-63), and neither
 * is its handle. */
class CUDAHandle
{
	struct Rep { lela_cuda_ctx *ctx; int refs; };
	Rep *_rep;

public:
	CUDAHandle () : _rep (new Rep)
	{
		_rep->refs = 1;
		_rep->ctx = 0;
		const char *d = std::getenv ("LELA_CUDA_DEVICE");
		int st = lela_cuda_create (&_rep->ctx, d ? std::atoi (d) : 0);
		if (st != LELA_CUDA_OK) {
			delete _rep;
			_rep = 0;
			throw LELAError ("CUDAModule: no usable B200 device (lela_cuda_create failed)");
		}
	}
	CUDAHandle (const CUDAHandle &h) : _rep (h._rep) { ++_rep->refs; }
	CUDAHandle &operator = (const CUDAHandle &h)
	{
		++h._rep->refs;
		release ();
		_rep = h._rep;
		return *this;
	}
	~CUDAHandle () { release (); }
	lela_cuda_ctx *get () const { return _rep->ctx; }

private:
	void release ()
	{
		if (_rep && --_rep->refs == 0) {
			lela_cuda_destroy (_rep->ctx);
			delete _rep;
		}
		_rep = 0;
	}
};

/** Throw the LELA exception that corresponds to a C ABI status. */
inline void lela_cuda_check (lela_cuda_ctx *ctx, int st, size_t aux = 0)
{
	switch (st) {
	case LELA_CUDA_OK: return;
	case LELA_CUDA_DIAG_NOT_INVERTIBLE: throw DiagonalEntryNotInvertible (aux);
	case LELA_CUDA_PIVOT_NOT_INVERTIBLE: throw LELAError ("Could not invert pivot-element in the ring");
	default: throw LELAError (lela_cuda_last_error (ctx));
	}
}

template <class Element>
struct CUDAModule;

/** The CUDA module over Modular<uint32>: GPU gemm, trsm and
 * Faugere-Lachartre; everything else is ZpModule<uint32>'s. */
template <>
struct CUDAModule<uint32> : public ZpModule<uint32>
{
	struct Tag { typedef ZpModule<uint32>::Tag Parent; };

	CUDAHandle cuda;

	CUDAModule (const Modular<uint32> &R) : ZpModule<uint32> (R) {}
};

namespace BLAS3
{

template <>
class _gemm<Modular<uint32>, CUDAModule<uint32>::Tag>
{
	template <class Modules, class Matrix1, class Matrix2, class Matrix3>
	static Matrix3 &gemm_impl (const Modular<uint32> &F, Modules &M, uint32 a, const Matrix1 &A, const Matrix2 &B, uint32 b, Matrix3 &C,
				   MatrixStorageTypes::Generic, MatrixStorageTypes::Generic, MatrixStorageTypes::Generic)
		{ return _gemm<Modular<uint32>, CUDAModule<uint32>::Tag::Parent>::op (F, M, a, A, B, b, C); }

	template <class Modules, class Matrix1, class Matrix2, class Matrix3>
	static Matrix3 &gemm_impl (const Modular<uint32> &F, Modules &M, uint32 a, const Matrix1 &A, const Matrix2 &B, uint32 b, Matrix3 &C,
				   MatrixStorageTypes::Dense, MatrixStorageTypes::Dense, MatrixStorageTypes::Dense)
	{
		lela_check (A.coldim () == B.rowdim ());
		lela_check (A.rowdim () == C.rowdim ());
		lela_check (B.coldim () == C.coldim ());
		size_t m = C.rowdim (), n = C.coldim (), k = A.coldim ();
		if (m == 0 || n == 0)
			return C;
		const uint32 *pa = k ? &A[0][0] : 0, *pb = k ? &B[0][0] : 0;
		int st = lela_cuda_gemm_zp_u32 (M.cuda.get (), m, n, k, F._modulus, a, pa, k ? A.disp () : 1,
						pb, k ? B.disp () : 1, b, &C[0][0], C.disp ());
		lela_cuda_check (M.cuda.get (), st);
		return C;
	}

public:
	template <class Modules, class Matrix1, class Matrix2, class Matrix3>
	static Matrix3 &op (const Modular<uint32> &F, Modules &M, uint32 a, const Matrix1 &A, const Matrix2 &B, uint32 b, Matrix3 &C)
		{ return gemm_impl (F, M, a, A, B, b, C,
				    typename Matrix1::StorageType (),
				    typename Matrix2::StorageType (),
				    typename Matrix3::StorageType ()); }
};

template <>
class _trsm<Modular<uint32>, CUDAModule<uint32>::Tag>
{
	template <class Modules, class Matrix1, class Matrix2>
	static Matrix2 &trsm_impl (const Modular<uint32> &F, Modules &M, uint32 a, const Matrix1 &A, Matrix2 &B,
				   TriangularMatrixType type, bool diagIsOne,
				   MatrixStorageTypes::Generic, MatrixStorageTypes::Generic)
		{ return _trsm<Modular<uint32>, CUDAModule<uint32>::Tag::Parent>::op (F, M, a, A, B, type, diagIsOne); }

	template <class Modules, class Matrix1, class Matrix2>
	static Matrix2 &trsm_impl (const Modular<uint32> &F, Modules &M, uint32 a, const Matrix1 &A, Matrix2 &B,
				   TriangularMatrixType type, bool diagIsOne,
				   MatrixStorageTypes::Dense, MatrixStorageTypes::Dense)
	{
		lela_check (A.coldim () == B.rowdim ());
		lela_check (A.rowdim () == B.rowdim ());
		size_t m = A.rowdim (), n = B.coldim ();
		if (m == 0)
			return B;
		size_t bad = 0;
		int st = lela_cuda_trsm_zp_u32 (M.cuda.get (), type == UpperTriangular, diagIsOne, m, n, F._modulus, a,
						&A[0][0], A.disp (), n ? &B[0][0] : 0, n ? B.disp () : 1, &bad);
		lela_cuda_check (M.cuda.get (), st, bad);
		return B;
	}

	// A stored by rows (SparseMatrix<uint32>), B dense: sparse rows of an
	// upper-triangular A go to the CSR solve (FaugereLachartre's A^-1 B,
	// lela/algorithms/faugere-lachartre.tcc:791); other rows and lower
	// triangular A go to the parent module.
	template <class Modules, class Matrix1, class Matrix2>
	static Matrix2 &trsm_impl (const Modular<uint32> &F, Modules &M, uint32 a, const Matrix1 &A, Matrix2 &B,
				   TriangularMatrixType type, bool diagIsOne,
				   MatrixStorageTypes::Rows, MatrixStorageTypes::Dense)
		{ return trsm_rows (F, M, a, A, B, type, diagIsOne,
				    typename VectorTraits<Modular<uint32>, typename Matrix1::ConstRow>::RepresentationType ()); }

	template <class Modules, class Matrix1, class Matrix2, class Rep>
	static Matrix2 &trsm_rows (const Modular<uint32> &F, Modules &M, uint32 a, const Matrix1 &A, Matrix2 &B,
				   TriangularMatrixType type, bool diagIsOne, Rep)
		{ return _trsm<Modular<uint32>, CUDAModule<uint32>::Tag::Parent>::op (F, M, a, A, B, type, diagIsOne); }

	template <class Modules, class Matrix1, class Matrix2>
	static Matrix2 &trsm_rows (const Modular<uint32> &F, Modules &M, uint32 a, const Matrix1 &A, Matrix2 &B,
				   TriangularMatrixType type, bool diagIsOne, VectorRepresentationTypes::Sparse)
	{
		if (type != UpperTriangular)
			return _trsm<Modular<uint32>, CUDAModule<uint32>::Tag::Parent>::op (F, M, a, A, B, type, diagIsOne);
		lela_check (A.coldim () == B.rowdim ());
		lela_check (A.rowdim () == B.rowdim ());
		const size_t m = A.rowdim (), n = B.coldim ();
		if (m == 0)
			return B;
		std::vector<uint64_t> rowptr (m + 1, 0);
		std::vector<uint32_t> colidx, vals;
		size_t i = 0;
		for (typename Matrix1::ConstRowIterator r = A.rowBegin (); r != A.rowEnd (); ++r, ++i) {
			for (typename Matrix1::ConstRow::const_iterator e = r->begin (); e != r->end (); ++e) {
				colidx.push_back ((uint32_t) (uint32) e->first);
				vals.push_back ((uint32_t) e->second);
			}
			rowptr[i + 1] = colidx.size ();
		}
		size_t bad = 0;
		int st = lela_cuda_trsm_csr_upper_zp_u32 (M.cuda.get (), m, n, F._modulus, a, diagIsOne, &rowptr[0],
							  colidx.empty () ? 0 : &colidx[0], vals.empty () ? 0 : &vals[0],
							  n ? &B[0][0] : 0, n ? B.disp () : 1, &bad);
		lela_cuda_check (M.cuda.get (), st, bad);
		return B;
	}

public:
	template <class Modules, class Matrix1, class Matrix2>
	static Matrix2 &op (const Modular<uint32> &F, Modules &M, uint32 a, const Matrix1 &A, Matrix2 &B,
			    TriangularMatrixType type, bool diagIsOne)
		{ return trsm_impl (F, M, a, A, B, type, diagIsOne,
				    typename Matrix1::StorageType (),
				    typename Matrix2::StorageType ()); }
};

} // namespace BLAS3

/** The CUDA module over Modular<uint8>, Modular<uint16>, Modular<float> and
 * Modular<double>: GPU gemm and trsm on dense operands (lela_cuda_gemm_zp,
 * lela_cuda_trsm_zp, which convert the elements to residues on the device
 * and back); everything else is ZpModule<Element>'s. */
template <class Element> struct CUDAElemCode;
template <> struct CUDAElemCode<uint8> { enum { value = LELA_CUDA_ELEM_U8 }; };
template <> struct CUDAElemCode<uint16> { enum { value = LELA_CUDA_ELEM_U16 }; };
template <> struct CUDAElemCode<float> { enum { value = LELA_CUDA_ELEM_F32 }; };
template <> struct CUDAElemCode<double> { enum { value = LELA_CUDA_ELEM_F64 }; };

template <class Element>
struct CUDAModule : public ZpModule<Element>
{
	struct Tag { typedef typename ZpModule<Element>::Tag Parent; };

	CUDAHandle cuda;

	CUDAModule (const Modular<Element> &R) : ZpModule<Element> (R) {}
};

/** A scalar of Modular<Element> as the residue the C ABI takes (the float
 * and double representatives can be negative). */
template <class Element>
inline uint32_t cuda_residue (const Modular<Element> &F, const Element &a)
{
	if (a < 0)
		return (uint32_t) ((long long) a + (long long) F._modulus);
	return (uint32_t) a;
}

namespace BLAS3
{

template <class Element>
class CUDAGemmElem
{
	typedef typename CUDAModule<Element>::Tag Tag;

	template <class Modules, class Matrix1, class Matrix2, class Matrix3>
	static Matrix3 &gemm_impl (const Modular<Element> &F, Modules &M, Element a, const Matrix1 &A, const Matrix2 &B, Element b, Matrix3 &C,
				   MatrixStorageTypes::Generic, MatrixStorageTypes::Generic, MatrixStorageTypes::Generic)
		{ return _gemm<Modular<Element>, typename Tag::Parent>::op (F, M, a, A, B, b, C); }

	template <class Modules, class Matrix1, class Matrix2, class Matrix3>
	static Matrix3 &gemm_impl (const Modular<Element> &F, Modules &M, Element a, const Matrix1 &A, const Matrix2 &B, Element b, Matrix3 &C,
				   MatrixStorageTypes::Dense, MatrixStorageTypes::Dense, MatrixStorageTypes::Dense)
	{
		lela_check (A.coldim () == B.rowdim ());
		lela_check (A.rowdim () == C.rowdim ());
		lela_check (B.coldim () == C.coldim ());
		size_t m = C.rowdim (), n = C.coldim (), k = A.coldim ();
		if (m == 0 || n == 0)
			return C;
		const Element *pa = k ? &A[0][0] : 0, *pb = k ? &B[0][0] : 0;
		int st = lela_cuda_gemm_zp (M.cuda.get (), CUDAElemCode<Element>::value, m, n, k,
					    (uint32_t) F._modulus, cuda_residue (F, a), pa, k ? A.disp () : 1,
					    pb, k ? B.disp () : 1, cuda_residue (F, b), &C[0][0], C.disp ());
		lela_cuda_check (M.cuda.get (), st);
		return C;
	}

public:
	template <class Modules, class Matrix1, class Matrix2, class Matrix3>
	static Matrix3 &op (const Modular<Element> &F, Modules &M, Element a, const Matrix1 &A, const Matrix2 &B, Element b, Matrix3 &C)
		{ return gemm_impl (F, M, a, A, B, b, C,
				    typename Matrix1::StorageType (),
				    typename Matrix2::StorageType (),
				    typename Matrix3::StorageType ()); }
};

template <class Element>
class CUDATrsmElem
{
	typedef typename CUDAModule<Element>::Tag Tag;

	template <class Modules, class Matrix1, class Matrix2>
	static Matrix2 &trsm_impl (const Modular<Element> &F, Modules &M, Element a, const Matrix1 &A, Matrix2 &B,
				   TriangularMatrixType type, bool diagIsOne,
				   MatrixStorageTypes::Generic, MatrixStorageTypes::Generic)
		{ return _trsm<Modular<Element>, typename Tag::Parent>::op (F, M, a, A, B, type, diagIsOne); }

	template <class Modules, class Matrix1, class Matrix2>
	static Matrix2 &trsm_impl (const Modular<Element> &F, Modules &M, Element a, const Matrix1 &A, Matrix2 &B,
				   TriangularMatrixType type, bool diagIsOne,
				   MatrixStorageTypes::Dense, MatrixStorageTypes::Dense)
	{
		lela_check (A.coldim () == B.rowdim ());
		lela_check (A.rowdim () == B.rowdim ());
		size_t m = A.rowdim (), n = B.coldim ();
		if (m == 0)
			return B;
		size_t bad = 0;
		int st = lela_cuda_trsm_zp (M.cuda.get (), CUDAElemCode<Element>::value, type == UpperTriangular, diagIsOne,
					    m, n, (uint32_t) F._modulus, cuda_residue (F, a), &A[0][0], A.disp (),
					    n ? &B[0][0] : 0, n ? B.disp () : 1, &bad);
		lela_cuda_check (M.cuda.get (), st, bad);
		return B;
	}

public:
	template <class Modules, class Matrix1, class Matrix2>
	static Matrix2 &op (const Modular<Element> &F, Modules &M, Element a, const Matrix1 &A, Matrix2 &B,
			    TriangularMatrixType type, bool diagIsOne)
		{ return trsm_impl (F, M, a, A, B, type, diagIsOne,
				    typename Matrix1::StorageType (),
				    typename Matrix2::StorageType ()); }
};

template <> class _gemm<Modular<uint8>, CUDAModule<uint8>::Tag> : public CUDAGemmElem<uint8> {};
template <> class _gemm<Modular<uint16>, CUDAModule<uint16>::Tag> : public CUDAGemmElem<uint16> {};
template <> class _gemm<Modular<float>, CUDAModule<float>::Tag> : public CUDAGemmElem<float> {};
template <> class _gemm<Modular<double>, CUDAModule<double>::Tag> : public CUDAGemmElem<double> {};
template <> class _trsm<Modular<uint8>, CUDAModule<uint8>::Tag> : public CUDATrsmElem<uint8> {};
template <> class _trsm<Modular<uint16>, CUDAModule<uint16>::Tag> : public CUDATrsmElem<uint16> {};
template <> class _trsm<Modular<float>, CUDAModule<float>::Tag> : public CUDATrsmElem<float> {};
template <> class _trsm<Modular<double>, CUDAModule<double>::Tag> : public CUDATrsmElem<double> {};

} // namespace BLAS3

/** The CUDA module over GF2: the GPU gemm on DenseMatrix<bool> operands
 * (LELA's packed rows: 64-bit words, LittleEndian bit order, the layout
 * without M4RI, lela/vector/bit-iterator.h:300-311); everything else is
 * GenericModule<GF2>'s. */
struct CUDAModuleGF2 : public GenericModule<GF2>
{
	struct Tag { typedef GenericModule<GF2>::Tag Parent; };

	CUDAHandle cuda;

	CUDAModuleGF2 (const GF2 &R) : GenericModule<GF2> (R) {}
};

namespace BLAS3
{

/** C <- a A B + b C over GF2 (replaces the generic Row*Row*Row gemm,
 * lela/blas/level3-generic.tcc:243-263).  DenseMatrix<bool> operands are
 * packed into contiguous words and go to lela_cuda_gemm_gf2; other matrix
 * types go to the parent module. */
template <>
class _gemm<GF2, CUDAModuleGF2::Tag>
{
	static void pack (const DenseMatrix<bool> &M, std::vector<uint64_t> &w)
	{
		const size_t words = (M.coldim () + 63) / 64;
		w.assign (M.rowdim () * words + 1, 0);
		size_t i = 0;
		for (DenseMatrix<bool>::ConstRowIterator r = M.rowBegin (); r != M.rowEnd (); ++r, ++i) {
			DenseMatrix<bool>::ConstRow::const_word_iterator it = r->word_begin ();
			for (size_t j = 0; j < words; ++j, ++it) {
				uint64_t v = *it;
				if (j == words - 1 && (M.coldim () & 63))
					v &= (~0ULL) >> (64 - (M.coldim () & 63));
				w[i * words + j] = v;
			}
		}
	}

	static void unpack (DenseMatrix<bool> &M, const std::vector<uint64_t> &w)
	{
		const size_t words = (M.coldim () + 63) / 64;
		size_t i = 0;
		for (DenseMatrix<bool>::RowIterator r = M.rowBegin (); r != M.rowEnd (); ++r, ++i) {
			DenseMatrix<bool>::Row::word_iterator it = r->word_begin ();
			for (size_t j = 0; j < words; ++j, ++it)
				*it = w[i * words + j];
		}
	}

public:
	template <class Modules, class Matrix1, class Matrix2, class Matrix3>
	static Matrix3 &op (const GF2 &F, Modules &M, bool a, const Matrix1 &A, const Matrix2 &B, bool b, Matrix3 &C)
		{ return _gemm<GF2, CUDAModuleGF2::Tag::Parent>::op (F, M, a, A, B, b, C); }

	template <class Modules>
	static DenseMatrix<bool> &op (const GF2 &F, Modules &M, bool a, const DenseMatrix<bool> &A,
				      const DenseMatrix<bool> &B, bool b, DenseMatrix<bool> &C)
	{
		lela_check (A.coldim () == B.rowdim ());
		lela_check (A.rowdim () == C.rowdim ());
		lela_check (B.coldim () == C.coldim ());
		const size_t m = C.rowdim (), n = C.coldim (), k = A.coldim ();
		if (m == 0 || n == 0)
			return C;
		std::vector<uint64_t> wa, wb, wc;
		pack (A, wa);
		pack (B, wb);
		pack (C, wc);
		const size_t kw = (k + 63) / 64, nw = (n + 63) / 64;
		int st = lela_cuda_gemm_gf2 (M.cuda.get (), m, n, k, a ? 1 : 0, &wa[0], kw ? kw : 1, &wb[0], nw,
					     b ? 1 : 0, &wc[0], nw);
		lela_cuda_check (M.cuda.get (), st);
		unpack (C, wc);
		return C;
	}
};

} // namespace BLAS3

/** FaugereLachartre over Modular<uint32> with the CUDA module: the same
 * interface as lela/algorithms/faugere-lachartre.h:40-82, the whole
 * pipeline on the GPU.  X is read row by row (any matrix type with sparse
 * rows: SparseMatrix<uint32>); R receives the result (resized to the
 * reference's shape when only_D is set). */
template <>
class FaugereLachartre<Modular<uint32>, CUDAModule<uint32> >
{
	Context<Modular<uint32>, CUDAModule<uint32> > &ctx;

public:
	FaugereLachartre (Context<Modular<uint32>, CUDAModule<uint32> > &_ctx) : ctx (_ctx) {}

	template <class Matrix>
	void echelonize (Matrix &R, const Matrix &X, size_t &rank, uint32 &det, bool reduced = true, bool only_D = false)
	{
		const size_t m = X.rowdim (), n = X.coldim ();
		std::vector<uint64_t> rowptr (m + 1, 0);
		std::vector<uint32_t> colidx, vals;
		size_t i = 0;
		for (typename Matrix::ConstRowIterator r = X.rowBegin (); r != X.rowEnd (); ++r, ++i) {
			for (typename Matrix::ConstRow::const_iterator e = r->begin (); e != r->end (); ++e) {
				colidx.push_back ((uint32_t) (uint32) e->first);
				vals.push_back ((uint32_t) e->second);
			}
			rowptr[i + 1] = colidx.size ();
		}
		// the result comes back as CSR rows (no dense m x n array); the
		// first guess of its size is twice X's entries, and a larger result
		// is fetched from the handle after the call
		std::vector<uint64_t> rrow (m + 1, 0);
		std::vector<uint32_t> rcol (2 * colidx.size () + 1), rval (2 * colidx.size () + 1);
		size_t rk = 0, rows = 0, bad = 0, nnz = 0;
		uint32_t d = 1;
		int st = lela_cuda_fl_echelonize_zp_u32_csr (ctx.M.cuda.get (), m, n, ctx.F._modulus, &rowptr[0],
							     colidx.empty () ? 0 : &colidx[0], vals.empty () ? 0 : &vals[0],
							     reduced, only_D, &rrow[0], &rcol[0], &rval[0], rcol.size (),
							     &nnz, &rk, &d, &rows, &bad);
		if (st == LELA_CUDA_ERR_CAPACITY) {
			rcol.resize (nnz);
			rval.resize (nnz);
			st = lela_cuda_fl_csr_fetch (ctx.M.cuda.get (), &rcol[0], &rval[0], nnz, 0);
		}
		rank = rk;
		det = d;
		if (st == LELA_CUDA_WRONG_MATRIX_FORM)
			throw WrongMatrixForm (bad);
		if (st == LELA_CUDA_DIAG_NOT_INVERTIBLE)
			return;  // the reference catches this and returns early (faugere-lachartre.tcc:790-799)
		lela_cuda_check (ctx.M.cuda.get (), st);
		if (only_D)
			R.resize (rows, n);
		i = 0;
		for (typename Matrix::RowIterator r = R.rowBegin (); r != R.rowEnd (); ++r, ++i) {
			r->clear ();
			if (i >= rows)
				continue;
			for (uint64_t e = rrow[i]; e < rrow[i + 1]; ++e)
				r->push_back (typename Matrix::Row::value_type (rcol[e], rval[e]));
		}
	}
};

/** EchelonForm over Modular<uint32> with the CUDA module: the interface and
 * the per-method control flow of lela/solutions/echelon-form.h:29-163.
 * Dense matrices go to the GPU for both Gauss-Jordan methods, reduced or
 * not: the asymptotically fast one (the default for a DenseMatrix; reduced,
 * the pivots keep their values) and the standard one (Elimination; reduced,
 * the pivots come out as 1).  The Faugere-Lachartre method runs the GPU
 * pipeline on a sparse copy of the rows.  Every other matrix type takes the
 * reference's Elimination on this context, as in the reference. */
template <>
class EchelonForm<Modular<uint32>, CUDAModule<uint32> >
{
	typedef Modular<uint32> Ring;
	typedef CUDAModule<uint32> Modules;

	Context<Ring, Modules> _ctx;
	Elimination<Ring, Modules> _elim;
	DenseMatrix<uint32> L;
	GaussJordan<Ring, Modules>::Permutation P;
	std::map<const void *, size_t> _rank_table;

	// reduced: 0 = non-reduced, 1 = pivots keep their values (Gauss-Jordan),
	// 2 = pivots 1 (Elimination)
	void gpu (DenseMatrix<uint32> &A, int reduced, size_t &rank)
	{
		size_t m = A.rowdim (), n = A.coldim ();
		uint32_t d = 1;
		rank = 0;
		if (m == 0 || n == 0)
			return;
		int st = reduced
			? lela_cuda_echelon_reduced_zp_u32 (_ctx.M.cuda.get (), m, n, _ctx.F._modulus, &A[0][0],
							    A.disp (), reduced == 2, &rank, &d)
			: lela_cuda_echelon_zp_u32 (_ctx.M.cuda.get (), m, n, _ctx.F._modulus, &A[0][0], A.disp (),
						    &rank, &d);
		lela_cuda_check (_ctx.M.cuda.get (), st);
	}

public:
	enum Method { METHOD_UNKNOWN, METHOD_STANDARD_GJ, METHOD_ASYMPTOTICALLY_FAST_GJ, METHOD_FAUGERE_LACHARTRE };

	EchelonForm (Context<Ring, Modules> &ctx) : _ctx (ctx), _elim (ctx) {}

	template <class Matrix>
	Matrix &echelonize (Matrix &A, bool reduced = false, Method method = METHOD_STANDARD_GJ)
	{
		size_t rank = 0;
		uint32 d;
		switch (method) {
		case METHOD_STANDARD_GJ:
			if (reduced)
				_elim.echelonize_reduced (A, L, P, rank, d, false);
			else
				_elim.echelonize (A, P, rank, d, false);
			break;
		case METHOD_FAUGERE_LACHARTRE:
			{
				FaugereLachartre<Ring, Modules> FL (_ctx);
				FL.echelonize (A, A, rank, d, reduced);
			}
			break;
		default:
			throw LELAError ("Invalid method for choice of matrix");
		}
		_rank_table[&A] = rank;
		return A;
	}

	DenseMatrix<uint32> &echelonize (DenseMatrix<uint32> &A, bool reduced = false, Method method = METHOD_ASYMPTOTICALLY_FAST_GJ)
	{
		size_t rank = 0;
		uint32 d;
		switch (method) {
		case METHOD_STANDARD_GJ:
			// Elimination: the non-reduced form equals Gauss-Jordan's
			// (tests/test-gauss-jordan.C:91-99); its reduced form has
			// unit pivots (lela/algorithms/elimination.tcc:222)
			gpu (A, reduced ? 2 : 0, rank);
			break;
		case METHOD_ASYMPTOTICALLY_FAST_GJ:
			gpu (A, reduced ? 1 : 0, rank);
			break;
		case METHOD_FAUGERE_LACHARTRE:
			{
				// the reference runs FL with its default (reduced) output here
				const size_t m = A.rowdim (), n = A.coldim ();
				SparseMatrix<uint32> X (m, n), R (m, n);
				for (size_t i = 0; i < m; ++i)
					for (size_t j = 0; j < n; ++j)
						if (A[i][j] != 0)
							X[i].push_back (SparseMatrix<uint32>::Row::value_type (j, A[i][j]));
				FaugereLachartre<Ring, Modules> FL (_ctx);
				FL.echelonize (R, X, rank, d);
				for (size_t i = 0; i < m; ++i) {
					for (size_t j = 0; j < n; ++j)
						A[i][j] = 0;
					for (SparseMatrix<uint32>::Row::const_iterator e = R[i].begin (); e != R[i].end (); ++e)
						A[i][e->first] = e->second;
				}
			}
			break;
		default:
			throw LELAError ("Invalid method for choice of matrix");
		}
		_rank_table[&A] = rank;
		return A;
	}

	template <class Matrix>
	size_t rank (const Matrix &A) const
	{
		std::map<const void *, size_t>::const_iterator it = _rank_table.find (&A);
		return it == _rank_table.end () ? 0 : it->second;
	}
};

} // namespace LELA

#endif /* LELA_CUDA_CUDA_MODULE_H */
