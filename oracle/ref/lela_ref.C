/* oracle/ref/lela_ref.C -- C entry points onto LELA's own CPU implementation.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is compiled (by oracle/Makefile)
 * together with the unmodified LELA headers and sources of the reference
 * tree into oracle/_ref/liblela_ref.so.  The library is the checker for the
 * CUDA path and the "reference" CPU baseline of bench.py; nothing in the
 * product (lela_b200/, include/) links or loads it.
 *
 * Every entry point copies plain row-major arrays into LELA's own matrix
 * types, runs the reference routine named in its comment through LELA's
 * public BLAS3 / algorithm interfaces, and copies the result back.
 */

#include <cstring>
#include <vector>
#include <pthread.h>
#include <algorithm>
#include <stdint.h>

#include "lela/ring/modular.h"
#include "lela/ring/gf2.h"
#include "lela/blas/context.h"
#include "lela/blas/level3.h"
#include "lela/matrix/dense.h"
#include "lela/matrix/sparse.h"
#include "lela/algorithms/faugere-lachartre.h"
#include "lela/algorithms/gauss-jordan.h"
#include "lela/algorithms/elimination.h"
#include "lela/util/error.h"
#include "lela/matrix/io.h"

#include <sstream>
#include <string>

using namespace LELA;

typedef Modular<uint32> Zp;

namespace {

void load_dense (DenseMatrix<uint32> &M, const uint32_t *src, size_t ld)
{
	for (size_t i = 0; i < M.rowdim (); ++i)
		std::memcpy (&M[i][0], src + i * ld, M.coldim () * sizeof (uint32_t));
}

void store_dense (const DenseMatrix<uint32> &M, uint32_t *dst, size_t ld)
{
	for (size_t i = 0; i < M.rowdim (); ++i)
		std::memcpy (dst + i * ld, &M[i][0], M.coldim () * sizeof (uint32_t));
}

template <class Modules>
void gemm_with (uint32_t p, size_t m, size_t n, size_t k, uint32_t a,
		const uint32_t *A, size_t lda, const uint32_t *B, size_t ldb,
		uint32_t b, uint32_t *C, size_t ldc)
{
	Zp F (p);
	Context<Zp, Modules> ctx (F);
	DenseMatrix<uint32> MA (m, k), MB (k, n), MC (m, n);
	if (m && k) load_dense (MA, A, lda);
	if (k && n) load_dense (MB, B, ldb);
	if (m && n) load_dense (MC, C, ldc);
	BLAS3::gemm (ctx, a, MA, MB, b, MC);
	if (m && n) store_dense (MC, C, ldc);
}

// GF(2) dense matrices: LELA's DenseMatrix<bool> rows are BitVector words,
// LittleEndian bit order (bit j of word w is column 64w+j).
void load_gf2 (DenseMatrix<bool> &M, const uint64_t *src, size_t ldw)
{
	size_t words = (M.coldim () + 63) / 64;
	size_t i = 0;
	for (DenseMatrix<bool>::RowIterator r = M.rowBegin (); r != M.rowEnd (); ++r, ++i) {
		DenseMatrix<bool>::Row::word_iterator w = r->word_begin ();
		for (size_t j = 0; j < words; ++j, ++w) {
			uint64_t v = src[i * ldw + j];
			if (j == words - 1 && (M.coldim () & 63))
				v &= (~0ULL) >> (64 - (M.coldim () & 63));
			*w = v;
		}
	}
}

void store_gf2 (const DenseMatrix<bool> &M, uint64_t *dst, size_t ldw)
{
	size_t words = (M.coldim () + 63) / 64;
	size_t i = 0;
	for (DenseMatrix<bool>::ConstRowIterator r = M.rowBegin (); r != M.rowEnd (); ++r, ++i) {
		DenseMatrix<bool>::ConstRow::const_word_iterator w = r->word_begin ();
		for (size_t j = 0; j < words; ++j, ++w)
			dst[i * ldw + j] = *w;
	}
}

// One slice of a process-parallel CPU run: kind 0 = gemm on a block of rows
// of A and C, kind 1 = trsm on a block of right-hand-side columns of B (C).
struct SliceJob {
	int kind; uint32_t p; size_t m, n, k; uint32_t a;
	const uint32_t *A; size_t lda; const uint32_t *B; size_t ldb;
	uint32_t b; uint32_t *C; size_t ldc; int upper, diag_is_one;
};

void *run_slice (void *arg)
{
	SliceJob *j = (SliceJob *) arg;
	if (j->kind == 0) {
		gemm_with<ZpModule<uint32> > (j->p, j->m, j->n, j->k, j->a, j->A, j->lda, j->B, j->ldb, j->b, j->C, j->ldc);
	} else {
		Zp F (j->p);
		Context<Zp, ZpModule<uint32> > ctx (F);
		DenseMatrix<uint32> MA (j->m, j->m), MB (j->m, j->n);
		load_dense (MA, j->A, j->lda);
		load_dense (MB, j->C, j->ldc);
		BLAS3::trsm (ctx, j->a, MA, MB, j->upper ? UpperTriangular : LowerTriangular, j->diag_is_one != 0);
		store_dense (MB, j->C, j->ldc);
	}
	return 0;
}

void run_jobs (std::vector<SliceJob> &jobs)
{
	std::vector<pthread_t> th (jobs.size ());
	for (size_t t = 0; t < jobs.size (); ++t) pthread_create (&th[t], 0, run_slice, &jobs[t]);
	for (size_t t = 0; t < jobs.size (); ++t) pthread_join (th[t], 0);
}

// Other element types of Modular<T> (lela/ring/modular.h:115-330).  A
// scalar given as a residue r becomes T's representative: r itself for the
// unsigned types, r or r - p (whichever lies in [-p/2, p/2]) for float and
// double, whose ModularTraits keep the symmetric range.
template <class T> T elem_of (uint32_t r, uint32_t p) { return (T) r; }
template <> float elem_of<float> (uint32_t r, uint32_t p)
	{ return 2ULL * r > p ? (float) ((long long) r - (long long) p) : (float) r; }
template <> double elem_of<double> (uint32_t r, uint32_t p)
	{ return 2ULL * r > p ? (double) ((long long) r - (long long) p) : (double) r; }

template <class T>
void load_t (DenseMatrix<T> &M, const T *src, size_t ld)
{
	for (size_t i = 0; i < M.rowdim (); ++i)
		for (size_t j = 0; j < M.coldim (); ++j)
			M[i][j] = src[i * ld + j];
}

template <class T>
void store_t (const DenseMatrix<T> &M, T *dst, size_t ld)
{
	for (size_t i = 0; i < M.rowdim (); ++i)
		for (size_t j = 0; j < M.coldim (); ++j)
			dst[i * ld + j] = M[i][j];
}

// BLAS3::gemm on Context<Modular<T> > (the default module stack).
template <class T>
void gemm_t (uint32_t p, size_t m, size_t n, size_t k, uint32_t a, const void *A, size_t lda,
	     const void *B, size_t ldb, uint32_t b, void *C, size_t ldc)
{
	Modular<T> F (p);
	Context<Modular<T> > ctx (F);
	DenseMatrix<T> MA (m, k), MB (k, n), MC (m, n);
	if (m && k) load_t (MA, (const T *) A, lda);
	if (k && n) load_t (MB, (const T *) B, ldb);
	if (m && n) load_t (MC, (const T *) C, ldc);
	BLAS3::gemm (ctx, elem_of<T> (a, p), MA, MB, elem_of<T> (b, p), MC);
	if (m && n) store_t (MC, (T *) C, ldc);
}

// BLAS3::trsm on Context<Modular<T> >; 1 with *bad_idx on
// DiagonalEntryNotInvertible (B then as LELA left it).
template <class T>
int trsm_t (uint32_t p, int upper, int diag_is_one, size_t m, size_t n, uint32_t a, const void *A,
	    size_t lda, void *B, size_t ldb, size_t *bad_idx)
{
	Modular<T> F (p);
	Context<Modular<T> > ctx (F);
	DenseMatrix<T> MA (m, m), MB (m, n);
	if (m) load_t (MA, (const T *) A, lda);
	if (m && n) load_t (MB, (const T *) B, ldb);
	int ret = 0;
	try {
		BLAS3::trsm (ctx, elem_of<T> (a, p), MA, MB, upper ? UpperTriangular : LowerTriangular, diag_is_one != 0);
	} catch (DiagonalEntryNotInvertible &e) {
		if (bad_idx) *bad_idx = e.idx ();
		ret = 1;
	}
	if (m && n) store_t (MB, (T *) B, ldb);
	return ret;
}

} // namespace

extern "C" {

/* BLAS3::gemm (lela/blas/level3.h:82) over Modular<uint32>.
 * module: 0 = ZpModule<uint32>, 1 = GenericModule, 2 = AllModules (the
 * default stack, Strassen-Winograd over ZpModule). */
int lela_ref_gemm_zp_u32 (int module, uint32_t p, size_t m, size_t n, size_t k, uint32_t a,
			  const uint32_t *A, size_t lda, const uint32_t *B, size_t ldb,
			  uint32_t b, uint32_t *C, size_t ldc)
{
	try {
		if (module == 0)
			gemm_with<ZpModule<uint32> > (p, m, n, k, a, A, lda, B, ldb, b, C, ldc);
		else if (module == 1)
			gemm_with<GenericModule<Zp> > (p, m, n, k, a, A, lda, B, ldb, b, C, ldc);
		else
			gemm_with<AllModules<Zp> > (p, m, n, k, a, A, lda, B, ldb, b, C, ldc);
	} catch (...) {
		return -1;
	}
	return 0;
}

/* Row-sliced, multi-threaded use of the same LELA routine: each thread runs
 * ZpModule gemm on its own block of rows of A and C with its own Context.
 * Z/p arithmetic is exact, so the result equals the single call. */
int lela_ref_gemm_zp_u32_threads (int nthreads, uint32_t p, size_t m, size_t n, size_t k, uint32_t a,
				  const uint32_t *A, size_t lda, const uint32_t *B, size_t ldb,
				  uint32_t b, uint32_t *C, size_t ldc)
{
	if (nthreads < 1) nthreads = 1;
	std::vector<SliceJob> jobs;
	size_t chunk = (m + nthreads - 1) / nthreads;
	for (int t = 0; t < nthreads; ++t) {
		size_t r0 = t * chunk, r1 = std::min (m, r0 + chunk);
		if (r0 >= r1) break;
		SliceJob j = { 0, p, r1 - r0, n, k, a, A + r0 * lda, lda, B, ldb, b, C + r0 * ldc, ldc, 0, 0 };
		jobs.push_back (j);
	}
	run_jobs (jobs);
	return 0;
}

/* BLAS3::trsm (lela/blas/level3.h:121) -> _trsm<.., GenericModule::Tag>
 * (lela/blas/level3-generic.tcc:421-498).  B <- a A^-1 B.
 * upper: 1 = UpperTriangular, 0 = LowerTriangular.
 * Returns 0, or 1 with *bad_idx set when LELA throws
 * DiagonalEntryNotInvertible(idx). */
int lela_ref_trsm_zp_u32 (uint32_t p, int upper, int diag_is_one, size_t m, size_t n, uint32_t a,
			  const uint32_t *A, size_t lda, uint32_t *B, size_t ldb, size_t *bad_idx)
{
	Zp F (p);
	Context<Zp, ZpModule<uint32> > ctx (F);
	DenseMatrix<uint32> MA (m, m), MB (m, n);
	if (m) load_dense (MA, A, lda);
	if (m && n) load_dense (MB, B, ldb);
	try {
		BLAS3::trsm (ctx, a, MA, MB, upper ? UpperTriangular : LowerTriangular, diag_is_one != 0);
	} catch (DiagonalEntryNotInvertible &e) {
		if (bad_idx) *bad_idx = e.idx ();
		if (m && n) store_dense (MB, B, ldb);
		return 1;
	}
	if (m && n) store_dense (MB, B, ldb);
	return 0;
}

/* Column-sliced, multi-threaded trsm: each thread solves its own block of
 * right-hand-side columns with the same LELA routine. */
int lela_ref_trsm_zp_u32_threads (int nthreads, uint32_t p, int upper, int diag_is_one, size_t m, size_t n,
				  uint32_t a, const uint32_t *A, size_t lda, uint32_t *B, size_t ldb)
{
	if (nthreads < 1) nthreads = 1;
	std::vector<SliceJob> jobs;
	size_t chunk = (n + nthreads - 1) / nthreads;
	for (int t = 0; t < nthreads; ++t) {
		size_t c0 = t * chunk, c1 = std::min (n, c0 + chunk);
		if (c0 >= c1) break;
		SliceJob j = { 1, p, m, c1 - c0, m, a, A, lda, 0, 0, 0, B + c0, ldb, upper, diag_is_one };
		jobs.push_back (j);
	}
	run_jobs (jobs);
	return 0;
}

/* Dense non-reduced row-echelon form as EchelonForm::echelonize does it for
 * a DenseMatrix (lela/solutions/echelon-form.h:103-134): GaussJordan::
 * echelonize (lela/algorithms/gauss-jordan.tcc:413-432) followed by
 * Elimination::move_L (lela/algorithms/elimination.tcc:372-391).
 * Also returns rank and det (product of the pivots). */
int lela_ref_echelon_zp_u32 (uint32_t p, size_t m, size_t n, uint32_t *A, size_t lda, size_t *rank, uint32_t *det)
{
	Zp F (p);
	Context<Zp> ctx (F);
	DenseMatrix<uint32> MA (m, n);
	if (m && n) load_dense (MA, A, lda);
	GaussJordan<Zp> GJ (ctx);
	Elimination<Zp> elim (ctx);
	GaussJordan<Zp>::Permutation P;
	size_t r = 0;
	Zp::Element d;
	try {
		GJ.echelonize (MA, P, r, d);
		elim.move_L (MA, MA);
	} catch (...) {
		return -1;
	}
	if (m && n) store_dense (MA, A, lda);
	*rank = r;
	/* GaussJordan's own det output is not the product of the pivots when
	 * the recursion meets zero column blocks; FaugereLachartre instead takes
	 * det from the leading entries of the echelon form (setup_splicer,
	 * lela/algorithms/faugere-lachartre.tcc:119), which is what is returned
	 * here. */
	Zp::Element pd = 1;
	for (size_t i = 0; i < r; ++i) {
		size_t c = 0;
		while (c < n && MA[i][c] == 0) ++c;
		if (c < n) F.mulin (pd, MA[i][c]);
	}
	*det = pd;
	(void) d;
	return 0;
}

/* Dense reduced row-echelon form as EchelonForm::echelonize (A, true) does
 * it for a DenseMatrix (lela/solutions/echelon-form.h:115-123): L sized
 * m x m, then GaussJordan::echelonize_reduced (lela/algorithms/
 * gauss-jordan.tcc:434-466), whose transform GaussJordanTransform
 * (:27-230) leaves every pivot at its value (no normalisation).  Rank and
 * det (product of the pivots, taken from the leading entries as above). */
int lela_ref_echelon_reduced_zp_u32 (uint32_t p, size_t m, size_t n, uint32_t *A, size_t lda, size_t *rank, uint32_t *det)
{
	Zp F (p);
	Context<Zp> ctx (F);
	DenseMatrix<uint32> MA (m, n);
	if (m && n) load_dense (MA, A, lda);
	GaussJordan<Zp> GJ (ctx);
	GaussJordan<Zp>::Permutation P;
	DenseMatrix<uint32> L (m, m);
	size_t r = 0;
	Zp::Element d;
	try {
		GJ.echelonize_reduced (MA, L, P, r, d);
	} catch (...) {
		return -1;
	}
	if (m && n) store_dense (MA, A, lda);
	*rank = r;
	Zp::Element pd = 1;
	for (size_t i = 0; i < r; ++i) {
		size_t c = 0;
		while (c < n && MA[i][c] == 0) ++c;
		if (c < n) F.mulin (pd, MA[i][c]);
	}
	*det = pd;
	(void) d;
	return 0;
}

/* The standard method's reduced form, EchelonForm::echelonize (A, true,
 * METHOD_STANDARD_GJ) on a DenseMatrix: Elimination::echelonize_reduced
 * (lela/algorithms/elimination.tcc:143-265) with the default pivot
 * strategy of a dense row (elimination.h:141-147) and no L, as
 * lela/solutions/echelon-form.h:111 calls it.  Each pivot row is scaled
 * by the inverse of its pivot (:222), so the pivots come out as 1.  det =
 * the product of the pivots before scaling. */
int lela_ref_elim_echelon_reduced_zp_u32 (uint32_t p, size_t m, size_t n, uint32_t *A, size_t lda, size_t *rank, uint32_t *det)
{
	Zp F (p);
	Context<Zp> ctx (F);
	DenseMatrix<uint32> MA (m, n);
	if (m && n) load_dense (MA, A, lda);
	Elimination<Zp> elim (ctx);
	Elimination<Zp>::Permutation P;
	DenseMatrix<uint32> L;
	size_t r = 0;
	Zp::Element d;
	try {
		elim.echelonize_reduced (MA, L, P, r, d, false);
	} catch (...) {
		return -1;
	}
	if (m && n) store_dense (MA, A, lda);
	*rank = r;
	*det = d;
	return 0;
}

/* Elimination::echelonize_reduced (A, L, P, rank, det, true) (lela/
 * algorithms/elimination.tcc:143-265) with the default pivot strategy of a
 * dense row: A <- its reduced form (pivots 1), L (m x m, dense) <- the
 * transform with A_out = L P A_in, P the row transpositions as pairs in the
 * reference's order (at most min(m, n)).  Returns 0, or -1 when a pivot is
 * not invertible. */
int lela_ref_elim_echelon_reduced_L_zp_u32 (uint32_t p, size_t m, size_t n, uint32_t *A, size_t lda, uint32_t *L, size_t ldl, size_t *P, size_t *np, size_t *rank, uint32_t *det)
{
	Zp F (p);
	Context<Zp> ctx (F);
	DenseMatrix<uint32> MA (m, n), ML (m, m);
	if (m && n) load_dense (MA, A, lda);
	Elimination<Zp> elim (ctx);
	Elimination<Zp>::Permutation PP;
	size_t r = 0;
	Zp::Element d;
	try {
		elim.echelonize_reduced (MA, ML, PP, r, d, true);
	} catch (...) {
		return -1;
	}
	if (m && n) store_dense (MA, A, lda);
	if (m) store_dense (ML, L, ldl);
	for (size_t k = 0; k < PP.size (); ++k) { P[2 * k] = PP[k].first; P[2 * k + 1] = PP[k].second; }
	*np = PP.size ();
	*rank = r;
	*det = d;
	return 0;
}

/* The non-reduced forms with L kept in A's lower part: gj = 0 runs
 * Elimination::echelonize (A, P, rank, det) with its default compute_L =
 * true (lela/algorithms/elimination.h:86-92, elimination.tcc:47-139: each
 * multiplier is written to (j, i) as the rows are eliminated); gj = 1 runs
 * GaussJordan::echelonize (A, P, rank, det) (lela/algorithms/
 * gauss-jordan.tcc:413-432, GaussTransform :232-411), which also leaves L
 * below the diagonal (gauss-jordan.h:92-104).  P as pairs in the
 * reference's order.  Returns 0, or -1 when a pivot is not invertible. */
int lela_ref_echelon_packed_L_zp_u32 (int gj, uint32_t p, size_t m, size_t n, uint32_t *A, size_t lda, size_t *P, size_t *np, size_t *rank, uint32_t *det)
{
	Zp F (p);
	Context<Zp> ctx (F);
	DenseMatrix<uint32> MA (m, n);
	if (m && n) load_dense (MA, A, lda);
	Elimination<Zp>::Permutation PP;
	size_t r = 0;
	Zp::Element d;
	try {
		if (gj) {
			GaussJordan<Zp> GJ (ctx);
			GJ.echelonize (MA, PP, r, d);
		} else {
			Elimination<Zp> elim (ctx);
			elim.echelonize (MA, PP, r, d);
		}
	} catch (...) {
		return -1;
	}
	if (m && n) store_dense (MA, A, lda);
	for (size_t k = 0; k < PP.size (); ++k) { P[2 * k] = PP[k].first; P[2 * k + 1] = PP[k].second; }
	*np = PP.size ();
	*rank = r;
	*det = d;
	return 0;
}

/* GaussJordan::echelonize_reduced (A, L, P, rank, det) (lela/algorithms/
 * gauss-jordan.tcc:434-466, through GaussJordanTransform :27-230): A <- its
 * reduced form (pivots keep their values), L (m x m, dense) <- the
 * transform with A_out = L P A_in, P the row transpositions as pairs in the
 * reference's order (at most min(m, n)).  det = the product of the pivots,
 * taken from the leading entries as lela_ref_echelon_reduced_zp_u32 does.
 * Returns 0, or -1 when a pivot is not invertible. */
int lela_ref_gj_echelon_reduced_L_zp_u32 (uint32_t p, size_t m, size_t n, uint32_t *A, size_t lda, uint32_t *L, size_t ldl, size_t *P, size_t *np, size_t *rank, uint32_t *det)
{
	Zp F (p);
	Context<Zp> ctx (F);
	DenseMatrix<uint32> MA (m, n), ML (m, m);
	if (m && n) load_dense (MA, A, lda);
	GaussJordan<Zp> GJ (ctx);
	GaussJordan<Zp>::Permutation PP;
	size_t r = 0;
	Zp::Element d;
	try {
		GJ.echelonize_reduced (MA, ML, PP, r, d);
	} catch (...) {
		return -1;
	}
	if (m && n) store_dense (MA, A, lda);
	if (m) store_dense (ML, L, ldl);
	for (size_t k = 0; k < PP.size (); ++k) { P[2 * k] = PP[k].first; P[2 * k + 1] = PP[k].second; }
	*np = PP.size ();
	*rank = r;
	Zp::Element pd = 1;
	for (size_t i = 0; i < r; ++i) {
		size_t c = 0;
		while (c < n && MA[i][c] == 0) ++c;
		if (c < n) F.mulin (pd, MA[i][c]);
	}
	*det = pd;
	(void) d;
	return 0;
}

/* Elimination::pluq (lela/algorithms/elimination.tcc:266-370) with the
 * default pivot strategy of a dense row: A <- L and U in place (L strictly
 * below the diagonal, unit diagonal implied), P and Q the row and column
 * transpositions in the order the reference returns them (reversed at its
 * end), as pairs in P[0..2*np), Q[0..2*nq).  The pair arrays hold at most
 * min(m, n) transpositions each.  Returns 0, or -1 when a pivot is not
 * invertible. */
int lela_ref_pluq_zp_u32 (uint32_t p, size_t m, size_t n, uint32_t *A, size_t lda, size_t *P, size_t *np, size_t *Q, size_t *nq, size_t *rank, uint32_t *det)
{
	Zp F (p);
	Context<Zp> ctx (F);
	DenseMatrix<uint32> MA (m, n);
	if (m && n) load_dense (MA, A, lda);
	Elimination<Zp> elim (ctx);
	Elimination<Zp>::Permutation PP, QQ;
	size_t r = 0;
	Zp::Element d;
	try {
		elim.pluq (MA, PP, QQ, r, d);
	} catch (...) {
		return -1;
	}
	if (m && n) store_dense (MA, A, lda);
	for (size_t k = 0; k < PP.size (); ++k) { P[2 * k] = PP[k].first; P[2 * k + 1] = PP[k].second; }
	for (size_t k = 0; k < QQ.size (); ++k) { Q[2 * k] = QQ[k].first; Q[2 * k + 1] = QQ[k].second; }
	*np = PP.size ();
	*nq = QQ.size ();
	*rank = r;
	*det = d;
	return 0;
}

/* Classical elimination Elimination::echelonize (lela/algorithms/
 * elimination.tcc:47-139), the reference's own cross-check for the
 * recursive GaussJordan result. */
int lela_ref_elim_echelon_zp_u32 (uint32_t p, size_t m, size_t n, uint32_t *A, size_t lda, size_t *rank, uint32_t *det)
{
	Zp F (p);
	Context<Zp> ctx (F);
	DenseMatrix<uint32> MA (m, n);
	if (m && n) load_dense (MA, A, lda);
	Elimination<Zp> elim (ctx);
	Elimination<Zp>::Permutation P;
	size_t r = 0;
	Zp::Element d;
	try {
		elim.echelonize (MA, P, r, d, DensePivotStrategy<Zp, AllModules<Zp> > (ctx), false);
	} catch (...) {
		return -1;
	}
	if (m && n) store_dense (MA, A, lda);
	*rank = r;
	*det = d;
	return 0;
}

/* FaugereLachartre::echelonize (lela/algorithms/faugere-lachartre.tcc:
 * 735-917) on a SparseMatrix<uint32> given in CSR form (rows sorted by
 * column).  R is returned dense row-major m x n (ldr), so callers can
 * compare it entry by entry.
 * Returns 0 = ok, 1 = WrongMatrixForm (the reference throws it from
 * setup_splicer, lela/algorithms/faugere-lachartre.tcc:80-81). */
int lela_ref_fl_echelonize_zp_u32 (uint32_t p, size_t m, size_t n,
				   const uint64_t *rowptr, const uint32_t *colidx, const uint32_t *vals,
				   int reduced, int only_D,
				   uint32_t *R, size_t ldr, size_t *rank, uint32_t *det, size_t *out_rows)
{
	Zp F (p);
	Context<Zp> ctx (F);
	typedef SparseMatrix<uint32> SM;
	SM X (m, n), Rm (m, n);
	size_t i = 0;
	for (SM::RowIterator r = X.rowBegin (); r != X.rowEnd (); ++r, ++i) {
		for (uint64_t e = rowptr[i]; e < rowptr[i + 1]; ++e)
			r->push_back (SM::Row::value_type (colidx[e], vals[e]));
	}
	FaugereLachartre<Zp> FL (ctx);
	size_t rk = 0;
	Zp::Element d;
	try {
		FL.echelonize (Rm, X, rk, d, reduced != 0, only_D != 0);
	} catch (WrongMatrixForm &e) {
		return 1;
	}
	size_t rows = Rm.rowdim ();
	for (size_t a = 0; a < rows; ++a)
		std::memset (R + a * ldr, 0, n * sizeof (uint32_t));
	i = 0;
	for (SM::ConstRowIterator r = Rm.rowBegin (); r != Rm.rowEnd (); ++r, ++i)
		for (SM::ConstRow::const_iterator e = r->begin (); e != r->end (); ++e)
			R[i * ldr + (size_t) (uint32_t) e->first] = (uint32_t) e->second;
	*rank = rk;
	*det = d;
	*out_rows = rows;
	return 0;
}

/* BLAS3::gemm over GF2 with DenseMatrix<bool> operands: AllModules<GF2>
 * without M4RI = StrassenModule over GenericModule (lela/ring/gf2.h:337-345),
 * i.e. the generic Row*Row*Row gemm (lela/blas/level3-generic.tcc:243-263). */
int lela_ref_gemm_gf2 (size_t m, size_t n, size_t k, int a,
		       const uint64_t *A, size_t lda, const uint64_t *B, size_t ldb,
		       int b, uint64_t *C, size_t ldc)
{
	GF2 F;
	Context<GF2> ctx (F);
	DenseMatrix<bool> MA (m, k), MB (k, n), MC (m, n);
	load_gf2 (MA, A, lda);
	load_gf2 (MB, B, ldb);
	load_gf2 (MC, C, ldc);
	BLAS3::gemm (ctx, a != 0, MA, MB, b != 0, MC);
	store_gf2 (MC, C, ldc);
	return 0;
}

/* GF(2) dense non-reduced echelon form: the EchelonForm dense path without
 * M4RI (GaussJordan + move_L), as for Modular<uint32>. */
int lela_ref_echelon_gf2 (size_t m, size_t n, uint64_t *A, size_t lda, size_t *rank)
{
	GF2 F;
	Context<GF2> ctx (F);
	DenseMatrix<bool> MA (m, n);
	load_gf2 (MA, A, lda);
	GaussJordan<GF2> GJ (ctx);
	Elimination<GF2> elim (ctx);
	GaussJordan<GF2>::Permutation P;
	size_t r = 0;
	bool d;
	try {
		GJ.echelonize (MA, P, r, d);
		elim.move_L (MA, MA);
	} catch (...) {
		return -1;
	}
	store_gf2 (MA, A, lda);
	*rank = r;
	return 0;
}

/* MatrixReader<Modular<uint32> >::detectFormat (lela/matrix/io.tcc:
 * 163-200) on the start of text: the FileFormatTag (lela/matrix/io.h:37-41)
 * as an int. */
int lela_ref_detect_format (const char *text)
{
	std::istringstream is (text);
	return (int) MatrixReader<Zp>::detectFormat (is);
}

/* MatrixReader::read (A, FORMAT_DUMAS) -> readDumas (lela/matrix/io.tcc:
 * 233-268) into a DenseMatrix<uint32> over Z/p.  *m, *n: the declared
 * size; the entries go to A (row stride n) when m * n <= cap.
 * Returns 0, 1 for InvalidMatrixInput, 2 for any other exception, 3 when
 * the matrix does not fit cap. */
int lela_ref_read_dumas (uint32_t p, const char *text, size_t cap, size_t *m, size_t *n, uint32_t *A)
{
	Zp F (p);
	MatrixReader<Zp> reader (F);
	DenseMatrix<uint32> M;
	std::istringstream is (text);
	try {
		reader.read (is, M, FORMAT_DUMAS);
	} catch (InvalidMatrixInput &) {
		return 1;
	} catch (...) {
		return 2;
	}
	*m = M.rowdim ();
	*n = M.coldim ();
	if (M.rowdim () * M.coldim () > cap)
		return 3;
	if (M.rowdim () && M.coldim ())
		store_dense (M, A, M.coldim ());
	return 0;
}

/* MatrixReader::read (A, format) into a DenseMatrix<uint32> already sized
 * m x n (the Turner, Matlab and Pretty readers do not resize; lela/matrix/
 * io.tcc:202-231, 295-341, 351-409).  Returns 0, 1 for InvalidMatrixInput,
 * 2 for any other exception; A (row stride n) receives the matrix. */
int lela_ref_read_matrix (int format, uint32_t p, const char *text, size_t m, size_t n, uint32_t *A)
{
	Zp F (p);
	MatrixReader<Zp> reader (F);
	DenseMatrix<uint32> M (m, n);
	std::istringstream is (text);
	try {
		reader.read (is, M, (FileFormatTag) format);
	} catch (InvalidMatrixInput &) {
		return 1;
	} catch (...) {
		return 2;
	}
	if (m && n)
		store_dense (M, A, n);
	return 0;
}

/* MatrixWriter::write (A, format) (lela/matrix/io.tcc:438-488 and the
 * writers after it) of a dense m x n matrix over Z/p; format is a
 * FileFormatTag (lela/matrix/io.h:37-41).  The text (NUL-terminated) goes
 * to buf when it fits cap bytes; *len = its length.  Returns 0, or 3 when
 * it does not fit. */
int lela_ref_write_matrix (int format, uint32_t p, size_t m, size_t n, const uint32_t *A, size_t lda, char *buf, size_t cap, size_t *len)
{
	Zp F (p);
	MatrixWriter<Zp> writer (F);
	DenseMatrix<uint32> M (m, n);
	if (m && n) load_dense (M, A, lda);
	std::ostringstream os;
	writer.write (os, M, (FileFormatTag) format);
	std::string t = os.str ();
	*len = t.size ();
	if (t.size () + 1 > cap)
		return 3;
	std::memcpy (buf, t.c_str (), t.size () + 1);
	return 0;
}

/* The same for FORMAT_DUMAS (writeDumas, io.tcc:526-534). */
int lela_ref_write_dumas (uint32_t p, size_t m, size_t n, const uint32_t *A, size_t lda, char *buf, size_t cap, size_t *len)
{
	Zp F (p);
	MatrixWriter<Zp> writer (F);
	DenseMatrix<uint32> M (m, n);
	if (m && n) load_dense (M, A, lda);
	std::ostringstream os;
	writer.write (os, M, FORMAT_DUMAS);
	std::string t = os.str ();
	*len = t.size ();
	if (t.size () + 1 > cap)
		return 3;
	std::memcpy (buf, t.c_str (), t.size () + 1);
	return 0;
}

/* BLAS3::gemm and BLAS3::trsm over Modular<uint8> (elem 1), Modular<uint16>
 * (2), Modular<float> (5) and Modular<double> (6) with the default module
 * stack (as tests/test-blas-zp-module.C:161-168 runs them).  Matrices hold
 * elements of that type; a and b are residues.  Returns -1 for an unknown
 * type or an exception other than DiagonalEntryNotInvertible. */
int lela_ref_gemm_zp_elem (int elem, uint32_t p, size_t m, size_t n, size_t k, uint32_t a,
			   const void *A, size_t lda, const void *B, size_t ldb, uint32_t b,
			   void *C, size_t ldc)
{
	try {
		switch (elem) {
		case 1: gemm_t<uint8> (p, m, n, k, a, A, lda, B, ldb, b, C, ldc); break;
		case 2: gemm_t<uint16> (p, m, n, k, a, A, lda, B, ldb, b, C, ldc); break;
		case 5: gemm_t<float> (p, m, n, k, a, A, lda, B, ldb, b, C, ldc); break;
		case 6: gemm_t<double> (p, m, n, k, a, A, lda, B, ldb, b, C, ldc); break;
		default: return -1;
		}
	} catch (...) {
		return -1;
	}
	return 0;
}

int lela_ref_trsm_zp_elem (int elem, uint32_t p, int upper, int diag_is_one, size_t m, size_t n,
			   uint32_t a, const void *A, size_t lda, void *B, size_t ldb, size_t *bad_idx)
{
	try {
		switch (elem) {
		case 1: return trsm_t<uint8> (p, upper, diag_is_one, m, n, a, A, lda, B, ldb, bad_idx);
		case 2: return trsm_t<uint16> (p, upper, diag_is_one, m, n, a, A, lda, B, ldb, bad_idx);
		case 5: return trsm_t<float> (p, upper, diag_is_one, m, n, a, A, lda, B, ldb, bad_idx);
		case 6: return trsm_t<double> (p, upper, diag_is_one, m, n, a, A, lda, B, ldb, bad_idx);
		default: return -1;
		}
	} catch (...) {
		return -1;
	}
}

} // extern "C"
