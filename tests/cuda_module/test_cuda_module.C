/* tests/cuda_module/test_cuda_module.C -- LELA code unchanged except for
 * the Modules type: the module-consistency pattern of the reference's own
 * tests (tests/test-blas-level3.h:1376-1461 testgemmConsistency, :1538-1604
 * testtrsmConsistency; tests/test-faugere-lachartre.C:179-247) with
 * Context<Modular<uint32>, CUDAModule<uint32>> against ZpModule/GenericModule.
 *
 * Built against the LELA headers (tests/cuda_module/build.sh) and run by
 * tests/test_cuda_module.py on a B200.  Exit status 0 = every check passed.
 */
#include <cstdio>
#include <vector>

#include "lela/ring/modular.h"
#include "lela/ring/gf2.h"
#include "lela/blas/context.h"
#include "lela/blas/level3.h"
#include "lela/matrix/dense.h"
#include "lela/matrix/sparse.h"
#include "lela/randiter/mersenne-twister.h"
#include "lela/algorithms/faugere-lachartre.h"
#include "lela/solutions/echelon-form.h"
#include "lela_cuda/cuda-module.h"

using namespace LELA;

typedef Modular<uint32> Zp;

static int failures = 0;

#define CHECK(cond, what) do { if (!(cond)) { std::printf ("FAIL: %s\n", what); ++failures; } \
	else std::printf ("ok:   %s\n", what); } while (0)

static void fill (DenseMatrix<uint32> &A, uint32 p, MersenneTwister &MT)
{
	for (size_t i = 0; i < A.rowdim (); ++i)
		for (size_t j = 0; j < A.coldim (); ++j)
			A.setEntry (i, j, MT.randomIntRange (0, p));
}

template <class M1, class M2>
static bool same (const M1 &A, const M2 &B)
{
	if (A.rowdim () != B.rowdim () || A.coldim () != B.coldim ())
		return false;
	for (size_t i = 0; i < A.rowdim (); ++i)
		for (size_t j = 0; j < A.coldim (); ++j) {
			uint32 a, b;
			A.getEntry (a, i, j);
			B.getEntry (b, i, j);
			if (a != b)
				return false;
		}
	return true;
}

static void test_gemm (uint32 p, size_t m, size_t n, size_t k, uint32 a, uint32 b)
{
	Zp F (p);
	Context<Zp, CUDAModule<uint32> > gpu (F);
	Context<Zp, ZpModule<uint32> > cpu (F);
	MersenneTwister MT (m * 31 + n * 7 + k);
	DenseMatrix<uint32> A (m, k), B (k, n), C (m, n), C2 (m, n);
	fill (A, p, MT); fill (B, p, MT); fill (C, p, MT);
	BLAS3::copy (cpu, C, C2);
	BLAS3::gemm (gpu, a, A, B, b, C);
	BLAS3::gemm (cpu, a, A, B, b, C2);
	char what[160];
	std::snprintf (what, sizeof what, "gemm p=%u %zux%zux%zu a=%u b=%u CUDAModule == ZpModule", p, m, n, k, a, b);
	CHECK (same (C, C2), what);

	// a submatrix view keeps the parent's stride (lela/matrix/dense.h:425-429)
	DenseMatrix<uint32> Cs (C, 1, 2, m - 2, n - 3), C2s (C2, 1, 2, m - 2, n - 3);
	DenseMatrix<uint32> As (A, 1, 0, m - 2, k);
	BLAS3::gemm (gpu, 3, As, DenseMatrix<uint32> (B, 0, 3, k, n - 3), 1, Cs);
	BLAS3::gemm (cpu, 3, As, DenseMatrix<uint32> (B, 0, 3, k, n - 3), 1, C2s);
	std::snprintf (what, sizeof what, "gemm on submatrix views p=%u", p);
	CHECK (same (C, C2), what);
}

static void test_trsm (uint32 p, size_t m, size_t n, bool upper, bool unit)
{
	Zp F (p);
	Context<Zp, CUDAModule<uint32> > gpu (F);
	Context<Zp, GenericModule<Zp> > cpu (F);
	MersenneTwister MT (m + 3 * n + upper);
	DenseMatrix<uint32> A (m, m), B (m, n), B2 (m, n);
	for (size_t i = 0; i < m; ++i)
		for (size_t j = 0; j < m; ++j) {
			bool in = upper ? j > i : j < i;
			A.setEntry (i, j, in ? MT.randomIntRange (0, p) : 0);
		}
	for (size_t i = 0; i < m; ++i)
		A.setEntry (i, i, unit ? 1 : MT.randomIntRange (1, p));
	fill (B, p, MT);
	BLAS3::copy (cpu, B, B2);
	BLAS3::trsm (gpu, 5, A, B, upper ? UpperTriangular : LowerTriangular, unit);
	BLAS3::trsm (cpu, 5, A, B2, upper ? UpperTriangular : LowerTriangular, unit);
	char what[160];
	std::snprintf (what, sizeof what, "trsm p=%u %zux%zu %s %s CUDAModule == GenericModule", p, m, n,
		       upper ? "upper" : "lower", unit ? "unit" : "non-unit");
	CHECK (same (B, B2), what);

	// a singular diagonal throws DiagonalEntryNotInvertible with LELA's index
	if (!unit && m > 10) {
		A.setEntry (3, 3, 0);
		A.setEntry (m - 4, m - 4, 0);
		size_t gi = (size_t) -1, ci = (size_t) -2;
		try { BLAS3::trsm (gpu, 1, A, B, upper ? UpperTriangular : LowerTriangular, false); }
		catch (DiagonalEntryNotInvertible e) { gi = e.idx (); }
		try { BLAS3::trsm (cpu, 1, A, B2, upper ? UpperTriangular : LowerTriangular, false); }
		catch (DiagonalEntryNotInvertible e) { ci = e.idx (); }
		std::snprintf (what, sizeof what, "trsm DiagonalEntryNotInvertible(%zu) == reference (%zu)", gi, ci);
		CHECK (gi == ci, what);
	}
}

// trsm with a sparse upper-triangular A (SparseMatrix<uint32>, the operand
// FaugereLachartre passes at faugere-lachartre.tcc:791): CUDAModule's CSR
// path against GenericModule on the same sparse rows, and the singular
// diagonal's index (a missing diagonal entry).
static void test_trsm_sparse (uint32 p, size_t m, size_t n)
{
	Zp F (p);
	Context<Zp, CUDAModule<uint32> > gpu (F);
	Context<Zp, GenericModule<Zp> > cpu (F);
	MersenneTwister MT (m * 5 + n);
	SparseMatrix<uint32> A (m, m);
	size_t i = 0;
	for (SparseMatrix<uint32>::RowIterator r = A.rowBegin (); r != A.rowEnd (); ++r, ++i) {
		r->push_back (SparseMatrix<uint32>::Row::value_type (i, MT.randomIntRange (1, p)));
		for (size_t j = i + 1; j < m; ++j)
			if (MT.randomDouble () < 0.05)
				r->push_back (SparseMatrix<uint32>::Row::value_type (j, MT.randomIntRange (1, p)));
	}
	DenseMatrix<uint32> B (m, n), B2 (m, n);
	fill (B, p, MT);
	BLAS3::copy (cpu, B, B2);
	BLAS3::trsm (gpu, 3, A, B, UpperTriangular, false);
	BLAS3::trsm (cpu, 3, A, B2, UpperTriangular, false);
	char what[160];
	std::snprintf (what, sizeof what, "trsm sparse upper p=%u %zux%zu CUDAModule == GenericModule", p, m, n);
	CHECK (same (B, B2), what);

	// drop two diagonal entries: DiagonalEntryNotInvertible with LELA's index
	SparseMatrix<uint32> S (m, m);
	i = 0;
	SparseMatrix<uint32>::ConstRowIterator ra = A.rowBegin ();
	for (SparseMatrix<uint32>::RowIterator r = S.rowBegin (); r != S.rowEnd (); ++r, ++ra, ++i)
		for (SparseMatrix<uint32>::ConstRow::const_iterator e = ra->begin (); e != ra->end (); ++e)
			if (!(e->first == i && (i == 5 || i == m - 7)))
				r->push_back (*e);
	size_t gi = (size_t) -1, ci = (size_t) -2;
	try { BLAS3::trsm (gpu, 1, S, B, UpperTriangular, false); }
	catch (DiagonalEntryNotInvertible e) { gi = e.idx (); }
	try { BLAS3::trsm (cpu, 1, S, B2, UpperTriangular, false); }
	catch (DiagonalEntryNotInvertible e) { ci = e.idx (); }
	std::snprintf (what, sizeof what, "trsm sparse DiagonalEntryNotInvertible(%zu) == reference (%zu)", gi, ci);
	CHECK (gi == ci, what);
}

// GF(2) gemm on DenseMatrix<bool>: CUDAModuleGF2 against GenericModule<GF2>.
static void test_gemm_gf2 (size_t m, size_t n, size_t k, bool a, bool b)
{
	GF2 F;
	Context<GF2, CUDAModuleGF2> gpu (F);
	Context<GF2, GenericModule<GF2> > cpu (F);
	MersenneTwister MT (m * 3 + n * 5 + k);
	DenseMatrix<bool> A (m, k), B (k, n), C (m, n), C2 (m, n);
	for (size_t i = 0; i < m; ++i)
		for (size_t j = 0; j < k; ++j)
			A.setEntry (i, j, MT.randomIntRange (0, 2) != 0);
	for (size_t i = 0; i < k; ++i)
		for (size_t j = 0; j < n; ++j)
			B.setEntry (i, j, MT.randomIntRange (0, 2) != 0);
	for (size_t i = 0; i < m; ++i)
		for (size_t j = 0; j < n; ++j) {
			bool v = MT.randomIntRange (0, 2) != 0;
			C.setEntry (i, j, v);
			C2.setEntry (i, j, v);
		}
	BLAS3::gemm (gpu, a, A, B, b, C);
	BLAS3::gemm (cpu, a, A, B, b, C2);
	bool eq = true;
	for (size_t i = 0; i < m && eq; ++i)
		for (size_t j = 0; j < n; ++j) {
			bool x, y;
			C.getEntry (x, i, j);
			C2.getEntry (y, i, j);
			if (x != y) { eq = false; break; }
		}
	char what[160];
	std::snprintf (what, sizeof what, "GF(2) gemm %zux%zux%zu a=%d b=%d CUDAModuleGF2 == GenericModule", m, n, k,
		       (int) a, (int) b);
	CHECK (eq, what);
}

// The reference test's F4 staircase (tests/test-faugere-lachartre.C:142-175),
// written here for SparseMatrix<uint32> rows.
static void random_f4 (SparseMatrix<uint32> &A, uint32 p, MersenneTwister &MT, double density)
{
	size_t col = 0, row = 0;
	for (SparseMatrix<uint32>::RowIterator r = A.rowBegin (); r != A.rowEnd (); ++r, ++row) {
		uint32 v = MT.randomIntRange (0, 7);
		if (v >= 1 && v <= 5) ++col;
		else if (v == 6) {
			size_t hi = A.coldim () - (A.rowdim () - row + 1);
			if (hi > col) col = MT.randomIntRange (col, hi);
		}
		if (col >= A.coldim ())
			break;
		r->push_back (SparseMatrix<uint32>::Row::value_type (col, MT.randomIntRange (1, p)));
		for (size_t j = col + 1; j < A.coldim (); ++j)
			if (MT.randomDouble () < density)
				r->push_back (SparseMatrix<uint32>::Row::value_type (j, MT.randomIntRange (1, p)));
	}
}

static void test_fl (uint32 p, size_t m, size_t n, bool reduced)
{
	Zp F (p);
	Context<Zp, CUDAModule<uint32> > gpu (F);
	Context<Zp> cpu (F);
	MersenneTwister MT (m * 13 + n);
	SparseMatrix<uint32> X (m, n), R1 (m, n), R2 (m, n);
	random_f4 (X, p, MT, 0.1);
	FaugereLachartre<Zp, CUDAModule<uint32> > FLg (gpu);
	FaugereLachartre<Zp> FLc (cpu);
	size_t r1 = 0, r2 = 0;
	uint32 d1 = 0, d2 = 0;
	FLg.echelonize (R1, X, r1, d1, reduced);
	FLc.echelonize (R2, X, r2, d2, reduced);
	char what[200];
	std::snprintf (what, sizeof what, "FaugereLachartre p=%u %zux%zu %s: R, rank (%zu/%zu), det (%u/%u) equal",
		       p, m, n, reduced ? "reduced" : "non-reduced", r1, r2, d1, d2);
	CHECK (r1 == r2 && d1 == d2 && BLAS3::equal (cpu, R1, R2), what);
}

// EchelonForm::echelonize on a DenseMatrix (lela/solutions/echelon-form.h:
// 103-150) under both contexts, per method and reduced flag: a
// rank-deficient matrix with a zero column, a zero row and dependent rows.
typedef EchelonForm<Zp, CUDAModule<uint32> > EFg;
typedef EchelonForm<Zp> EFc;

static void test_echelon (uint32 p, size_t m, size_t n, bool reduced, int method)
{
	Zp F (p);
	Context<Zp, CUDAModule<uint32> > gpu (F);
	Context<Zp> cpu (F);
	MersenneTwister MT (m * 7 + n + method);
	DenseMatrix<uint32> A (m, n), B (m, n);
	fill (A, p, MT);
	for (size_t i = 0; i < m; ++i)
		A.setEntry (i, 1, 0);
	for (size_t j = 0; j < n; ++j) {
		A.setEntry (2, j, 0);
		A.setEntry (m - 1, j, (A[0][j] * (uint64_t) 3) % p);
		A.setEntry (m - 2, j, (A[3][j] + (uint64_t) A[4][j]) % p);
	}
	BLAS3::copy (cpu, A, B);
	EFg Eg (gpu);
	EFc Ec (cpu);
	Eg.echelonize (A, reduced, (EFg::Method) method);
	Ec.echelonize (B, reduced, (EFc::Method) method);
	// the reference's EchelonForm::rank does not compile when instantiated
	// (operator[] on its const map, echelon-form.h:163): count B's rows
	size_t rb = 0;
	for (size_t i = 0; i < m; ++i)
		for (size_t j = 0; j < n; ++j)
			if (B[i][j] != 0) { ++rb; break; }
	char what[200];
	std::snprintf (what, sizeof what, "EchelonForm p=%u %zux%zu %s method %d: form and rank (%zu/%zu) equal",
		       p, m, n, reduced ? "reduced" : "non-reduced", method, Eg.rank (A), rb);
	CHECK (Eg.rank (A) == rb && BLAS3::equal (cpu, A, B), what);
}

// The other element types (tests/test-blas-zp-module.C:161-168): gemm and
// trsm with Context<Modular<T>, CUDAModule<T> > against the default module
// stack of Modular<T> (odd moduli: the representatives are unique).
template <class T>
static void fill_t (const Modular<T> &F, DenseMatrix<T> &A, MersenneTwister &MT, bool nonzero = false)
{
	for (size_t i = 0; i < A.rowdim (); ++i)
		for (size_t j = 0; j < A.coldim (); ++j) {
			T x;
			F.init (x, (integer) MT.randomIntRange (nonzero ? 1 : 0, (uint32) F._modulus));
			A.setEntry (i, j, x);
		}
}

template <class T>
static bool same_t (const DenseMatrix<T> &A, const DenseMatrix<T> &B)
{
	for (size_t i = 0; i < A.rowdim (); ++i)
		for (size_t j = 0; j < A.coldim (); ++j)
			if (A[i][j] != B[i][j])
				return false;
	return true;
}

template <class T>
static void test_elem (const char *name, uint32 p, size_t m, size_t n, size_t k)
{
	Modular<T> F (p);
	Context<Modular<T>, CUDAModule<T> > gpu (F);
	Context<Modular<T> > cpu (F);
	MersenneTwister MT (p + m);
	DenseMatrix<T> A (m, k), B (k, n), C (m, n), C2 (m, n);
	fill_t (F, A, MT); fill_t (F, B, MT); fill_t (F, C, MT);
	BLAS3::copy (cpu, C, C2);
	T a, b;
	F.init (a, (integer) 3);
	F.init (b, (integer) (p - 1));
	BLAS3::gemm (gpu, a, A, B, b, C);
	BLAS3::gemm (cpu, a, A, B, b, C2);
	char what[160];
	std::snprintf (what, sizeof what, "gemm %s p=%u %zux%zux%zu CUDAModule == default modules", name, p, m, n, k);
	CHECK (same_t (C, C2), what);

	DenseMatrix<T> L (m, m), X (m, n), X2 (m, n);
	for (size_t i = 0; i < m; ++i)
		for (size_t j = 0; j < m; ++j) {
			T x;
			F.init (x, (integer) (j < i ? MT.randomIntRange (0, p) : (j == i ? MT.randomIntRange (1, p) : 0)));
			L.setEntry (i, j, x);
		}
	fill_t (F, X, MT);
	BLAS3::copy (cpu, X, X2);
	BLAS3::trsm (gpu, a, L, X, LowerTriangular, false);
	BLAS3::trsm (cpu, a, L, X2, LowerTriangular, false);
	std::snprintf (what, sizeof what, "trsm %s p=%u %zux%zu lower CUDAModule == default modules", name, p, m, n);
	CHECK (same_t (X, X2), what);
}

int main ()
{
	try {
		test_gemm (65521, 130, 257, 300, 1, 1);
		test_gemm (2147483647u, 100, 90, 513, 7, 11);
		test_gemm (251, 64, 64, 64, 250, 0);
		test_trsm (65521, 130, 40, true, false);
		test_trsm (65521, 130, 40, false, false);
		test_trsm (2147483647u, 70, 9, true, true);
		test_trsm (2147483647u, 70, 9, false, true);
		test_gemm_gf2 (130, 200, 257, true, true);
		test_gemm_gf2 (64, 70, 129, true, false);
		test_trsm_sparse (65521, 300, 40);
		test_trsm_sparse (2147483647u, 90, 7);
		test_fl (65521, 96, 128, true);
		test_fl (65521, 96, 128, false);
		test_fl (2147483647u, 200, 300, true);
		test_echelon (65521, 90, 130, false, EFc::METHOD_ASYMPTOTICALLY_FAST_GJ);
		test_echelon (65521, 90, 130, true, EFc::METHOD_ASYMPTOTICALLY_FAST_GJ);
		test_echelon (251, 140, 70, true, EFc::METHOD_ASYMPTOTICALLY_FAST_GJ);
		test_echelon (65521, 90, 130, false, EFc::METHOD_STANDARD_GJ);
		test_echelon (65521, 60, 80, true, EFc::METHOD_STANDARD_GJ);
		test_echelon (251, 140, 70, true, EFc::METHOD_STANDARD_GJ);
		test_elem<uint8> ("Modular<uint8>", 251, 50, 30, 50);
		test_elem<uint16> ("Modular<uint16>", 65521, 50, 30, 50);
		test_elem<float> ("Modular<float>", 2039, 50, 30, 50);
		test_elem<float> ("Modular<float>", 4093, 70, 20, 90);
		test_elem<double> ("Modular<double>", 33554393, 50, 30, 50);
		test_elem<double> ("Modular<double>", 67108859, 70, 20, 90);
	} catch (LELAError &e) {
		std::printf ("FAIL: LELAError thrown\n");
		return 2;
	}
	std::printf (failures ? "%d FAILURES\n" : "all passed\n", failures);
	return failures ? 1 : 0;
}
