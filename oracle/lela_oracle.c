/* oracle/lela_oracle.c -- CPU restatement of LELA's exact linear-algebra hot
 * path (see lela_oracle.h).  TEST INFRASTRUCTURE ONLY: never linked into the
 * product; it is the checker the CUDA path is compared against.
 *
 * Citations are to files of the LELA source tree.
 */
#define _POSIX_C_SOURCE 200809L
#include "lela_oracle.h"
#include <stdlib.h>
#include <string.h>
#include <pthread.h>

/* ---------------------------------------------------------------- Z/p -- */

/* 2^64 mod p, as ZpModule<uint32>::init_two_64 computes it
 * (lela/ring/modular.h:604-626): six squarings of 2. */
static uint32_t two_64_mod (uint32_t p)
{
	uint64_t t = 2;
	for (int i = 0; i < 6; ++i)
		t = (t * t) % p;
	return (uint32_t) t;
}

/* Delayed-reduction dot product of _dot<Modular<uint32>, ZpModule>
 * (lela/blas/level1-modular.tcc:135-158): a 64-bit running sum of 32x32-bit
 * products; on wrap-around 2^64 mod p is added back; one final % p. */
static uint32_t dot_zp (uint32_t p, uint32_t two64, const uint32_t *x, size_t incx,
			const uint32_t *y, size_t incy, size_t k)
{
	uint64_t s = 0, t;
	for (size_t l = 0; l < k; ++l) {
		t = (uint64_t) x[l * incx] * (uint64_t) y[l * incy];
		s += t;
		if (s < t)
			s += two64;
	}
	return (uint32_t) (s % p);
}

static uint32_t mulmod (uint32_t p, uint32_t x, uint32_t y)
{
	return (uint32_t) (((uint64_t) x * y) % p);
}

/* Modular<uint32>::axpyin (lela/ring/modular.h:527-532): r <- a*x + r. */
static uint32_t axpy_mod (uint32_t p, uint32_t r, uint32_t a, uint32_t x)
{
	return (uint32_t) (((uint64_t) a * x + r) % p);
}

/* Modular<uint32>::eea (lela/ring/modular.h:540-557) in its EEAElement
 * type, which is a 32-bit int for uint32 elements (modular.h:210): every
 * intermediate wraps modulo 2^32 exactly as the reference's arithmetic does.
 * For p < 2^31 this is the textbook extended Euclidean algorithm; for
 * p >= 2^31 the modulus itself wraps negative and the reference's inverse
 * fails (or returns what the wrapped arithmetic yields), and so does this. */
static void eea32 (int32_t *gcd, int32_t *a, int32_t x, int32_t *b, int32_t y)
{
	if (y == 0) {
		*gcd = x; *a = 1; *b = 0;
	} else {
		int32_t q, r;
		if (y == -1) { q = (int32_t) (0u - (uint32_t) x); r = 0; }
		else { q = x / y; r = x % y; }
		eea32 (gcd, b, y, a, r);
		*b = (int32_t) ((uint32_t) *b - (uint32_t) q * (uint32_t) *a);
	}
}

/* Modular<uint32>::inv (lela/ring/modular.h:460-474): eea on (y, p) as
 * 32-bit ints; on gcd == 1 the coefficient is shifted up by p if negative
 * (shift_up, :228-229), converted to uint32 and shifted down once if >= p
 * (shift_down, :230-232).  Returns 0 when the reference reports failure. */
uint32_t oracle_inv_zp (uint32_t p, uint32_t x)
{
	int32_t gcd, ty, tm;
	eea32 (&gcd, &ty, (int32_t) x, &tm, (int32_t) p);
	if (gcd != 1)
		return 0;
	if (ty < 0)
		ty = (int32_t) ((uint32_t) ty + p);
	uint32_t r = (uint32_t) ty;
	if ((uint64_t) r >= (uint64_t) p)
		r -= p;
	return r;
}

/* Generic gemm, Row x Col case (lela/blas/level3-generic.tcc:285-322): one
 * delayed-reduction dot per entry, then C(i,j) <- b*C(i,j) + a*d
 * (Modular::mulin then axpyin). */
static void gemm_rows (uint32_t p, uint32_t two64, size_t r0, size_t r1, size_t n, size_t k, uint32_t a,
		       const uint32_t *A, size_t lda, const uint32_t *B, size_t ldb,
		       uint32_t b, uint32_t *C, size_t ldc)
{
	for (size_t i = r0; i < r1; ++i)
		for (size_t j = 0; j < n; ++j) {
			uint32_t d = dot_zp (p, two64, A + i * lda, 1, B + j, ldb, k);
			uint32_t c = mulmod (p, C[i * ldc + j], b);
			C[i * ldc + j] = axpy_mod (p, c, a, d);
		}
}

int oracle_gemm_zp_u32 (uint32_t p, size_t m, size_t n, size_t k, uint32_t a,
			const uint32_t *A, size_t lda, const uint32_t *B, size_t ldb,
			uint32_t b, uint32_t *C, size_t ldc)
{
	gemm_rows (p, two_64_mod (p), 0, m, n, k, a, A, lda, B, ldb, b, C, ldc);
	return 0;
}

struct gemm_job {
	uint32_t p, two64; size_t r0, r1, n, k; uint32_t a;
	const uint32_t *A; size_t lda; const uint32_t *B; size_t ldb;
	uint32_t b; uint32_t *C; size_t ldc;
};

static void *gemm_job_run (void *arg)
{
	struct gemm_job *j = (struct gemm_job *) arg;
	gemm_rows (j->p, j->two64, j->r0, j->r1, j->n, j->k, j->a, j->A, j->lda, j->B, j->ldb, j->b, j->C, j->ldc);
	return NULL;
}

int oracle_gemm_zp_u32_threads (int nthreads, uint32_t p, size_t m, size_t n, size_t k, uint32_t a,
				const uint32_t *A, size_t lda, const uint32_t *B, size_t ldb,
				uint32_t b, uint32_t *C, size_t ldc)
{
	if (nthreads < 1) nthreads = 1;
	if (nthreads > 256) nthreads = 256;
	pthread_t th[256];
	struct gemm_job jobs[256];
	size_t chunk = (m + nthreads - 1) / nthreads;
	int used = 0;
	for (int t = 0; t < nthreads; ++t) {
		size_t r0 = t * chunk, r1 = r0 + chunk < m ? r0 + chunk : m;
		if (r0 >= r1) break;
		struct gemm_job j = { p, two_64_mod (p), r0, r1, n, k, a, A, lda, B, ldb, b, C, ldc };
		jobs[used] = j;
		pthread_create (&th[used], NULL, gemm_job_run, &jobs[used]);
		++used;
	}
	for (int t = 0; t < used; ++t)
		pthread_join (th[t], NULL);
	return 0;
}

/* Recursive trsm of _trsm<Ring, GenericModule::Tag>::trsm_impl
 * (lela/blas/level3-generic.tcc:421-498) for dense operands (align = 1):
 * split at l = rows/2; lower: solve A11, B2 <- a*B2 - A21*B1, solve A22
 * with coefficient 1; upper: solve A22, B1 <- a*B1 - A12*B2, solve A11.
 * Leaf: scale the row by a*A(0,0)^-1 or report DiagonalEntryNotInvertible;
 * indices are re-based by l on the way up (:461-467, :478-489). */
static int trsm_rec (uint32_t p, uint32_t two64, int upper, int diag_is_one, size_t m, size_t n, uint32_t a,
		     const uint32_t *A, size_t lda, uint32_t *B, size_t ldb, size_t *bad_idx)
{
	if (m == 0)
		return 0;
	if (a == 0) {
		for (size_t i = 0; i < m; ++i)
			memset (B + i * ldb, 0, n * sizeof (uint32_t));
		return 0;
	}
	if (m == 1) {
		uint32_t s = a;
		if (!diag_is_one) {
			uint32_t ai = oracle_inv_zp (p, A[0]);
			if (ai == 0) { *bad_idx = 0; return 1; }
			s = mulmod (p, ai, a);
		}
		for (size_t j = 0; j < n; ++j)
			B[j] = mulmod (p, B[j], s);
		return 0;
	}
	size_t l = m / 2;
	const uint32_t *A11 = A, *A12 = A + l, *A21 = A + l * lda, *A22 = A + l * lda + l;
	uint32_t *B1 = B, *B2 = B + l * ldb;
	uint32_t minus_one = p - 1;
	int rc;
	if (!upper) {
		if ((rc = trsm_rec (p, two64, upper, diag_is_one, l, n, a, A11, lda, B1, ldb, bad_idx)))
			return rc;
		gemm_rows (p, two64, 0, m - l, n, l, minus_one, A21, lda, B1, ldb, a, B2, ldb);
		if ((rc = trsm_rec (p, two64, upper, diag_is_one, m - l, n, 1, A22, lda, B2, ldb, bad_idx))) {
			*bad_idx += l;
			return rc;
		}
	} else {
		if ((rc = trsm_rec (p, two64, upper, diag_is_one, m - l, n, a, A22, lda, B2, ldb, bad_idx))) {
			*bad_idx += l;
			return rc;
		}
		gemm_rows (p, two64, 0, l, n, m - l, minus_one, A12, lda, B2, ldb, a, B1, ldb);
		if ((rc = trsm_rec (p, two64, upper, diag_is_one, l, n, 1, A11, lda, B1, ldb, bad_idx)))
			return rc;
	}
	return 0;
}

int oracle_trsm_zp_u32 (uint32_t p, int upper, int diag_is_one, size_t m, size_t n, uint32_t a,
			const uint32_t *A, size_t lda, uint32_t *B, size_t ldb, size_t *bad_idx)
{
	size_t idx = 0;
	int rc = trsm_rec (p, two_64_mod (p), upper, diag_is_one, m, n, a, A, lda, B, ldb, &idx);
	if (rc && bad_idx)
		*bad_idx = idx;
	return rc;
}

/* Classical elimination, Elimination::echelonize (lela/algorithms/
 * elimination.tcc:47-139) with DensePivotStrategy (lela/algorithms/
 * pivot-strategy.tcc:19-42): for row i, scan columns from the current one
 * and, within a column, rows from i downwards; the first nonzero is the
 * pivot; swap it into row i (a transposition), multiply det by it, add
 * -a/x times row i to every row below with a nonzero a in the pivot column.
 * Pivots are not normalised.  GaussJordan::echelonize + move_L produces the
 * same matrix (tests/test-gauss-jordan.C:91-99). */
int oracle_echelon_zp_u32 (uint32_t p, size_t m, size_t n, uint32_t *A, size_t lda,
			   size_t *rank, uint32_t *det)
{
	size_t i = 0, col = 0;
	uint32_t d = 1 % p;
	uint32_t *tmp = (uint32_t *) malloc ((n ? n : 1) * sizeof (uint32_t));
	for (; i < m && col < n; ++i, ++col) {
		size_t prow = m;
		for (; col < n; ++col) {
			for (size_t r = i; r < m; ++r)
				if (A[r * lda + col] != 0) { prow = r; break; }
			if (prow < m) break;
		}
		if (prow == m)
			break;
		if (prow != i) {
			memcpy (tmp, A + i * lda, n * sizeof (uint32_t));
			memcpy (A + i * lda, A + prow * lda, n * sizeof (uint32_t));
			memcpy (A + prow * lda, tmp, n * sizeof (uint32_t));
		}
		uint32_t x = A[i * lda + col];
		d = mulmod (p, d, x);
		uint32_t xinv = oracle_inv_zp (p, x);
		if (xinv == 0) { free (tmp); return -1; }
		uint32_t negxinv = (p - xinv) % p;
		for (size_t r = i + 1; r < m; ++r) {
			uint32_t av = A[r * lda + col];
			if (av == 0) continue;
			uint32_t f = mulmod (p, av, negxinv);
			for (size_t c = col; c < n; ++c)
				A[r * lda + c] = axpy_mod (p, A[r * lda + c], f, A[i * lda + c]);
		}
	}
	free (tmp);
	*rank = i;
	*det = d;
	return 0;
}

/* Reduced row-echelon form, GaussJordan::echelonize_reduced (lela/
 * algorithms/gauss-jordan.tcc:434-466) through GaussJordanTransform
 * (:27-230), as EchelonForm::echelonize (A, true) runs it on a dense
 * matrix.  The recursion takes the columns left to right; in each it picks
 * the first nonzero at or below the current row of the column as reduced
 * by the earlier pivot rows -- the pivot rows and pivot values of the
 * non-reduced form above -- and clears the column in every other row by
 * adding multiples of the pivot row, whose entry keeps its value (:74-107:
 * a_ii is set back, the transform's diagonal stays one).  So every pivot
 * row of the result is its non-reduced row plus multiples of the later
 * pivot rows, zero in their pivot columns, which determines it.  Restated
 * as the non-reduced form followed by clearing upwards, the bottom pivot
 * row first: R_j <- R_j - (R_j[c_i] / x_i) R_i for j < i. */
int oracle_echelon_reduced_zp_u32 (uint32_t p, size_t m, size_t n, uint32_t *A, size_t lda,
				   size_t *rank, uint32_t *det)
{
	int rc = oracle_echelon_zp_u32 (p, m, n, A, lda, rank, det);
	if (rc)
		return rc;
	size_t r = *rank;
	size_t *pc = (size_t *) malloc ((r ? r : 1) * sizeof (size_t));
	for (size_t i = 0; i < r; ++i) {
		size_t c = 0;
		while (A[i * lda + c] == 0)
			++c;
		pc[i] = c;
	}
	for (size_t i = r; i-- > 0;) {
		/* every pivot was inverted by the form above */
		uint32_t negxinv = (p - oracle_inv_zp (p, A[i * lda + pc[i]])) % p;
		for (size_t j = 0; j < i; ++j) {
			uint32_t a = A[j * lda + pc[i]];
			if (a == 0)
				continue;
			uint32_t f = mulmod (p, a, negxinv);
			for (size_t c = pc[i]; c < n; ++c)
				A[j * lda + c] = axpy_mod (p, A[j * lda + c], f, A[i * lda + c]);
		}
	}
	free (pc);
	return 0;
}

/* The standard method's reduced form, Elimination::echelonize_reduced
 * (lela/algorithms/elimination.tcc:143-265), as EchelonForm::echelonize
 * (A, true, METHOD_STANDARD_GJ) runs it.  Row i: the first nonzero at or
 * below it in the current column of the matrix reduced by the earlier
 * pivot rows (the same pivots as above), scaled by the inverse of its pivot
 * (:222), then cleared from every other row.  The result is the form above
 * with each pivot row divided by its pivot; det is the product of the
 * pivots before scaling. */
int oracle_echelon_reduced_unit_zp_u32 (uint32_t p, size_t m, size_t n, uint32_t *A, size_t lda,
					size_t *rank, uint32_t *det)
{
	int rc = oracle_echelon_reduced_zp_u32 (p, m, n, A, lda, rank, det);
	if (rc)
		return rc;
	for (size_t i = 0; i < *rank; ++i) {
		size_t c = 0;
		while (A[i * lda + c] == 0)
			++c;
		uint32_t xinv = oracle_inv_zp (p, A[i * lda + c]);
		for (; c < n; ++c)
			A[i * lda + c] = mulmod (p, A[i * lda + c], xinv);
	}
	return 0;
}

/* The standard method's reduced form with its transform,
 * Elimination::echelonize_reduced (A, L, P, rank, det, true) (lela/
 * algorithms/elimination.tcc:143-265), step by step as the reference takes
 * it.  L (m x m, leading dimension ldl) starts as the identity (:176-184).
 * Step i: the first column from the current one with a nonzero at or below
 * row i, and its first such row; when that row is not i, rows i and it are
 * swapped in A, and in L both rows and columns (:203-210), and the pair is
 * recorded; det is multiplied by the pivot x; row i of A and of L is scaled
 * by 1/x (:221-227); every other row j with a nonzero a in the pivot column
 * gets row j <- row j - a row i, in A and in L (:229-244).  So at the end
 * A = L P A_in, P the transpositions applied in order.  P holds them as
 * pairs in the reference's order (not reversed).  Returns 0, or -1 when a
 * pivot is not invertible (the reference throws). */
static int echelon_reduced_L (uint32_t p, size_t m, size_t n, uint32_t *A, size_t lda,
			      uint32_t *L, size_t ldl, size_t *P, size_t *np,
			      size_t *rank, uint32_t *det, uint32_t *pivots)
{
	size_t i, c, npp = 0;
	uint32_t d = 1 % p;
	for (i = 0; i < m; ++i)
		for (c = 0; c < m; ++c)
			L[i * ldl + c] = (i == c) ? 1 % p : 0;
	size_t pc = 0;
	for (i = 0; i < m && pc < n; ++i, ++pc) {
		size_t prow = m;
		for (; pc < n; ++pc) {
			for (size_t r = i; r < m; ++r)
				if (A[r * lda + pc] != 0) { prow = r; break; }
			if (prow < m) break;
		}
		if (prow == m)
			break;
		if (prow != i) {
			for (c = 0; c < n; ++c) {
				uint32_t t = A[i * lda + c];
				A[i * lda + c] = A[prow * lda + c];
				A[prow * lda + c] = t;
			}
			for (c = 0; c < m; ++c) {
				uint32_t t = L[i * ldl + c];
				L[i * ldl + c] = L[prow * ldl + c];
				L[prow * ldl + c] = t;
			}
			for (c = 0; c < m; ++c) {
				uint32_t t = L[c * ldl + i];
				L[c * ldl + i] = L[c * ldl + prow];
				L[c * ldl + prow] = t;
			}
			P[2 * npp] = i; P[2 * npp + 1] = prow; ++npp;
		}
		uint32_t x = A[i * lda + pc];
		d = mulmod (p, d, x);
		if (pivots)
			pivots[i] = x;
		uint32_t xinv = oracle_inv_zp (p, x);
		if (xinv == 0)
			return -1;
		for (c = 0; c < n; ++c)
			A[i * lda + c] = mulmod (p, A[i * lda + c], xinv);
		for (c = 0; c < m; ++c)
			L[i * ldl + c] = mulmod (p, L[i * ldl + c], xinv);
		for (size_t j = 0; j < m; ++j) {
			uint32_t a = A[j * lda + pc];
			if (j == i || a == 0)
				continue;
			uint32_t nega = (p - a) % p;
			for (c = 0; c < n; ++c)
				A[j * lda + c] = axpy_mod (p, A[j * lda + c], nega, A[i * lda + c]);
			for (c = 0; c < m; ++c)
				L[j * ldl + c] = axpy_mod (p, L[j * ldl + c], nega, L[i * ldl + c]);
		}
	}
	*np = npp;
	*rank = i;
	*det = d;
	return 0;
}

int oracle_echelon_reduced_L_zp_u32 (uint32_t p, size_t m, size_t n, uint32_t *A, size_t lda,
				     uint32_t *L, size_t ldl, size_t *P, size_t *np,
				     size_t *rank, uint32_t *det)
{
	return echelon_reduced_L (p, m, n, A, lda, L, ldl, P, np, rank, det, NULL);
}

/* The fast method's reduced form with its transform,
 * GaussJordan::echelonize_reduced (A, L, P, rank, det) (lela/algorithms/
 * gauss-jordan.tcc:434-466) through GaussJordanTransform (:27-230).  The
 * recursion takes the same pivots and transpositions, in the same order, as
 * the standard method above; its leaf clears the pivot column in every
 * other row and writes the multipliers into the transform's column k, but
 * leaves the pivot row and the transform's diagonal entry as they are
 * (:74-107).  So the result differs from the standard method's only in the
 * pivot rows: R_i and L_i of the fast method are x_i R_i and x_i L_i of the
 * standard one (x_i the i-th pivot), which is how it is restated here.
 * Returns 0, or -1 when a pivot is not invertible. */
int oracle_gj_echelon_reduced_L_zp_u32 (uint32_t p, size_t m, size_t n, uint32_t *A, size_t lda,
					uint32_t *L, size_t ldl, size_t *P, size_t *np,
					size_t *rank, uint32_t *det)
{
	size_t k = m < n ? m : n;
	uint32_t *x = (uint32_t *) malloc ((k ? k : 1) * sizeof (uint32_t));
	int rc = echelon_reduced_L (p, m, n, A, lda, L, ldl, P, np, rank, det, x);
	if (rc == 0)
		for (size_t i = 0; i < *rank; ++i) {
			for (size_t c = 0; c < n; ++c)
				A[i * lda + c] = mulmod (p, A[i * lda + c], x[i]);
			for (size_t c = 0; c < m; ++c)
				L[i * ldl + c] = mulmod (p, L[i * ldl + c], x[i]);
		}
	free (x);
	return rc;
}

/* GaussTransform's d (lela/algorithms/gauss-jordan.tcc:232-411) over the
 * column range [c0, c1), from the pivots alone: a block with no pivot
 * copies d_0 into d (:243-247: the block is zero), a one-column block
 * multiplies d by its pivot (:259), and a wider block runs its left half
 * with d_0 into d_1 = 1 and its right half with d_1 as d_0 into d
 * (:300-343).  pcol[] (increasing) and pval[] are the r pivots. */
static uint32_t gj_det_rec (uint32_t p, size_t c0, size_t c1, uint32_t d0, uint32_t d,
			    const size_t *pcol, const uint32_t *pval, size_t r)
{
	size_t lo = 0, hi = r;
	while (lo < hi) {  /* first pivot column >= c0 */
		size_t mid = (lo + hi) / 2;
		if (pcol[mid] < c0) lo = mid + 1; else hi = mid;
	}
	if (lo == r || pcol[lo] >= c1)
		return d0;
	if (c1 - c0 == 1)
		return mulmod (p, d, pval[lo]);
	size_t m1 = (c1 - c0) / 2;
	uint32_t d1 = gj_det_rec (p, c0, c0 + m1, d0, 1 % p, pcol, pval, r);
	return gj_det_rec (p, c0 + m1, c1, d1, d, pcol, pval, r);
}

/* The non-reduced forms that keep L below the diagonal of A.
 * gj = 0: Elimination::echelonize (A, P, rank, det) with its default
 * compute_L = true (lela/algorithms/elimination.h:86-92, elimination.tcc:
 * 47-139), step by step: the pivot rule and transpositions as above; every
 * row j below with a nonzero a in the pivot column gets row j <- row j +
 * (-a/x) row i over the whole row (the L entries left of column i included,
 * :113), then (j, i) <- -a/x (:115-116).  det = product of the pivots.
 * gj = 1: GaussJordan::echelonize (A, P, rank, det) (gauss-jordan.tcc:
 * 413-432): the same A and P (its transform stores the same multipliers),
 * and GaussTransform's d (gj_det_rec).  P as pairs in the order applied.
 * Returns 0, or -1 when a pivot is not invertible. */
int oracle_echelon_packed_L_zp_u32 (int gj, uint32_t p, size_t m, size_t n, uint32_t *A,
				    size_t lda, size_t *P, size_t *np, size_t *rank, uint32_t *det)
{
	size_t k = m < n ? m : n, i, c, npp = 0, pc = 0;
	size_t *pcol = (size_t *) malloc ((k ? k : 1) * sizeof (size_t));
	uint32_t *pval = (uint32_t *) malloc ((k ? k : 1) * sizeof (uint32_t));
	uint32_t d = 1 % p;
	int rc = 0;
	for (i = 0; i < m && pc < n; ++i, ++pc) {
		size_t prow = m;
		for (; pc < n; ++pc) {
			for (size_t r = i; r < m; ++r)
				if (A[r * lda + pc] != 0) { prow = r; break; }
			if (prow < m) break;
		}
		if (prow == m)
			break;
		if (prow != i) {
			for (c = 0; c < n; ++c) {
				uint32_t t = A[i * lda + c];
				A[i * lda + c] = A[prow * lda + c];
				A[prow * lda + c] = t;
			}
			P[2 * npp] = i; P[2 * npp + 1] = prow; ++npp;
		}
		uint32_t x = A[i * lda + pc];
		pcol[i] = pc;
		pval[i] = x;
		d = mulmod (p, d, x);
		uint32_t xinv = oracle_inv_zp (p, x);
		if (xinv == 0) { rc = -1; break; }
		uint32_t negxinv = (p - xinv) % p;
		for (size_t j = i + 1; j < m; ++j) {
			uint32_t a = A[j * lda + pc];
			if (a == 0)
				continue;
			uint32_t f = mulmod (p, a, negxinv);
			for (c = 0; c < n; ++c)
				A[j * lda + c] = axpy_mod (p, A[j * lda + c], f, A[i * lda + c]);
			A[j * lda + i] = f;
		}
	}
	if (rc == 0) {
		*np = npp;
		*rank = i;
		*det = gj ? gj_det_rec (p, 0, n, 1 % p, 1 % p, pcol, pval, i) : d;
	}
	free (pcol);
	free (pval);
	return rc;
}

/* PLUQ decomposition, Elimination::pluq (lela/algorithms/elimination.tcc:
 * 266-370) with DensePivotStrategy (lela/algorithms/pivot-strategy.tcc:
 * 19-42).  Step i: the first column from i on, in the current column
 * order, with a nonzero at or below row i, and its first such row; that row
 * and that column are swapped into place (transpositions (i, row) and (i,
 * col)), det is multiplied by the pivot x, and every row j below with a
 * nonzero a in column i gets row j <- row j - (a / x) row i right of column
 * i and L entry a / x in column i.  Stops when no pivot is left or i
 * reaches the column count.  P and Q are returned reversed, as the
 * reference returns them (:362-363), as pairs. */
int oracle_pluq_zp_u32 (uint32_t p, size_t m, size_t n, uint32_t *A, size_t lda,
			size_t *P, size_t *np, size_t *Q, size_t *nq, size_t *rank, uint32_t *det)
{
	size_t i, npp = 0, nqq = 0;
	uint32_t d = 1 % p;
	for (i = 0; i < m && i < n; ++i) {
		size_t prow = m, pcol = i;
		for (; pcol < n; ++pcol) {
			for (size_t r = i; r < m; ++r)
				if (A[r * lda + pcol] != 0) { prow = r; break; }
			if (prow < m) break;
		}
		if (prow == m)
			break;
		if (prow != i) {
			for (size_t c = 0; c < n; ++c) {
				uint32_t t = A[i * lda + c];
				A[i * lda + c] = A[prow * lda + c];
				A[prow * lda + c] = t;
			}
			P[2 * npp] = i; P[2 * npp + 1] = prow; ++npp;
		}
		if (pcol != i) {
			for (size_t r = 0; r < m; ++r) {
				uint32_t t = A[r * lda + i];
				A[r * lda + i] = A[r * lda + pcol];
				A[r * lda + pcol] = t;
			}
			Q[2 * nqq] = i; Q[2 * nqq + 1] = pcol; ++nqq;
		}
		uint32_t x = A[i * lda + i];
		d = mulmod (p, d, x);
		uint32_t xinv = oracle_inv_zp (p, x);
		if (xinv == 0)
			return -1;
		uint32_t negxinv = (p - xinv) % p;
		for (size_t j = i + 1; j < m; ++j) {
			uint32_t a = A[j * lda + i];
			if (a == 0)
				continue;
			uint32_t f = mulmod (p, a, negxinv);
			for (size_t c = i + 1; c < n; ++c)
				A[j * lda + c] = axpy_mod (p, A[j * lda + c], f, A[i * lda + c]);
			A[j * lda + i] = (p - f) % p;
		}
	}
	for (size_t k = 0; k < npp / 2; ++k)
		for (int h = 0; h < 2; ++h) {
			size_t t = P[2 * k + h]; P[2 * k + h] = P[2 * (npp - 1 - k) + h]; P[2 * (npp - 1 - k) + h] = t;
		}
	for (size_t k = 0; k < nqq / 2; ++k)
		for (int h = 0; h < 2; ++h) {
			size_t t = Q[2 * k + h]; Q[2 * k + h] = Q[2 * (nqq - 1 - k) + h]; Q[2 * (nqq - 1 - k) + h] = t;
		}
	*np = npp;
	*nq = nqq;
	*rank = i;
	*det = d;
	return 0;
}

/* Faugere-Lachartre (lela/algorithms/faugere-lachartre.tcc:735-917).
 *
 * setup_splicer (:47-146) walks the rows: the head of a sparse row is its
 * first stored entry (BLAS1::head, lela/blas/level1-generic.tcc:452-460); a
 * head larger than the last pivot column makes a pivot row and multiplies
 * det by the head value; an equal head makes a non-pivot row; a smaller one
 * throws WrongMatrixForm(row); the first empty row stops the walk and every
 * row from there on is a non-pivot row.  The matrix is cut into A (pivot
 * rows x pivot columns, upper triangular), B (pivot rows x other columns),
 * C and D (non-pivot rows); then B <- A^-1 B (trsm, :791), D <- D - C B
 * (gemm, :805), D <- echelon(D) (:822), whose pivots multiply det and add
 * to the rank (:833-834).  The reduced variant (:851-902) splits D into
 * D1 | D2 by D's pivot columns, D2 <- D1^-1 D2, B2 <- B2 - B1 D2, and
 * writes the reduced echelon form; rows come out ordered by pivot column
 * with the zero rows last.
 */
int oracle_fl_echelonize_zp_u32 (uint32_t p, size_t m, size_t n,
				 const uint64_t *rowptr, const uint32_t *colidx, const uint32_t *vals,
				 int reduced, int only_D,
				 uint32_t *R, size_t ldr, size_t *rank, uint32_t *det,
				 size_t *out_rows, size_t *bad_row)
{
	uint32_t d = 1 % p;
	long last_col = -1;
	size_t npiv = 0, row;
	char *is_piv_row = (char *) calloc (m ? m : 1, 1);
	char *is_piv_col = (char *) calloc (n ? n : 1, 1);
	for (row = 0; row < m; ++row) {
		if (rowptr[row] == rowptr[row + 1])
			break;
		long col = colidx[rowptr[row]];
		uint32_t a = vals[rowptr[row]];
		if (col == last_col)
			; /* non-pivot row */
		else if (col < last_col) {
			free (is_piv_row); free (is_piv_col);
			if (bad_row) *bad_row = row;
			return 1;
		} else {
			is_piv_row[row] = 1;
			is_piv_col[col] = 1;
			last_col = col;
			++npiv;
		}
		d = mulmod (p, d, a);
	}

	size_t nres = n - npiv, mres = m - npiv;
	size_t *piv_rows = (size_t *) malloc ((npiv + 1) * sizeof (size_t));
	size_t *res_rows = (size_t *) malloc ((mres + 1) * sizeof (size_t));
	size_t *piv_cols = (size_t *) malloc ((npiv + 1) * sizeof (size_t));
	size_t *res_cols = (size_t *) malloc ((nres + 1) * sizeof (size_t));
	long *col_pos = (long *) malloc ((n + 1) * sizeof (long));
	size_t a_ = 0, b_ = 0;
	for (size_t r = 0; r < m; ++r) { if (is_piv_row[r]) piv_rows[a_++] = r; else res_rows[b_++] = r; }
	a_ = b_ = 0;
	for (size_t c = 0; c < n; ++c) {
		if (is_piv_col[c]) { col_pos[c] = (long) a_; piv_cols[a_++] = c; }
		else { col_pos[c] = (long) b_; res_cols[b_++] = c; }
	}

	uint32_t *A = (uint32_t *) calloc (npiv * npiv + 1, 4);
	uint32_t *B = (uint32_t *) calloc (npiv * nres + 1, 4);
	uint32_t *C = (uint32_t *) calloc (mres * npiv + 1, 4);
	uint32_t *D = (uint32_t *) calloc (mres * nres + 1, 4);
	for (size_t i = 0; i < npiv; ++i) {
		size_t r = piv_rows[i];
		for (uint64_t e = rowptr[r]; e < rowptr[r + 1]; ++e) {
			size_t c = colidx[e];
			if (is_piv_col[c]) A[i * npiv + col_pos[c]] = vals[e];
			else B[i * nres + col_pos[c]] = vals[e];
		}
	}
	for (size_t i = 0; i < mres; ++i) {
		size_t r = res_rows[i];
		for (uint64_t e = rowptr[r]; e < rowptr[r + 1]; ++e) {
			size_t c = colidx[e];
			if (is_piv_col[c]) C[i * npiv + col_pos[c]] = vals[e];
			else D[i * nres + col_pos[c]] = vals[e];
		}
	}

	int status = 0;
	size_t bad = 0;
	if (oracle_trsm_zp_u32 (p, 1, 0, npiv, nres, 1, A, npiv, B, nres, &bad)) {
		status = 2;
		goto out;
	}
	oracle_gemm_zp_u32 (p, mres, nres, npiv, p - 1, C, npiv, B, nres, 1, D, nres);

	size_t rd = 0;
	uint32_t dd = 1;
	if (oracle_echelon_zp_u32 (p, mres, nres, D, nres, &rd, &dd)) { status = 3; goto out; }
	/* setup_splicer on the echelon form of D: dense heads are first
	 * nonzeros (lela/blas/level1-generic.tcc:434-446). */
	size_t *dpiv = (size_t *) malloc ((rd + 1) * sizeof (size_t));
	char *is_dpiv = (char *) calloc (nres + 1, 1);
	for (size_t i = 0; i < rd; ++i) {
		size_t c = 0;
		while (c < nres && D[i * nres + c] == 0) ++c;
		dpiv[i] = c;
		is_dpiv[c] = 1;
		d = mulmod (p, d, D[i * nres + c]);
	}
	*rank = npiv + rd;
	*det = d;

	/* Global output: per row, its leading column and a writer. */
	if (reduced) {
		size_t nrem = nres - rd;
		size_t *rem = (size_t *) malloc ((nrem + 1) * sizeof (size_t));
		size_t *dpos = (size_t *) malloc ((nres + 1) * sizeof (size_t));
		for (size_t c = 0, a2 = 0, b2 = 0; c < nres; ++c) {
			if (is_dpiv[c]) dpos[c] = a2++; else { dpos[c] = b2; rem[b2++] = c; }
		}
		uint32_t *D1 = (uint32_t *) calloc (rd * rd + 1, 4);
		uint32_t *D2 = (uint32_t *) calloc (rd * nrem + 1, 4);
		for (size_t i = 0; i < rd; ++i)
			for (size_t c = 0; c < nres; ++c) {
				if (is_dpiv[c]) D1[i * rd + dpos[c]] = D[i * nres + c];
				else D2[i * nrem + dpos[c]] = D[i * nres + c];
			}
		oracle_trsm_zp_u32 (p, 1, 0, rd, nrem, 1, D1, rd, D2, nrem, &bad);
		size_t rows_out;
		if (only_D) {
			rows_out = rd;
			for (size_t i = 0; i < rd; ++i) {
				uint32_t *Ri = R + i * ldr;
				memset (Ri, 0, n * 4);
				Ri[res_cols[dpiv[i]]] = 1;
				for (size_t c = 0; c < nrem; ++c) Ri[res_cols[rem[c]]] = D2[i * nrem + c];
			}
		} else {
			uint32_t *B1 = (uint32_t *) calloc (npiv * rd + 1, 4);
			uint32_t *B2 = (uint32_t *) calloc (npiv * nrem + 1, 4);
			for (size_t i = 0; i < npiv; ++i)
				for (size_t c = 0; c < nres; ++c) {
					if (is_dpiv[c]) B1[i * rd + dpos[c]] = B[i * nres + c];
					else B2[i * nrem + dpos[c]] = B[i * nres + c];
				}
			oracle_gemm_zp_u32 (p, npiv, nrem, rd, p - 1, B1, rd, D2, nrem, 1, B2, nrem);
			rows_out = m;
			/* merge the X pivots and the D pivots by leading column */
			size_t xi = 0, di = 0, out = 0;
			while (xi < npiv || di < rd) {
				size_t xc = xi < npiv ? piv_cols[xi] : (size_t) -1;
				size_t dc = di < rd ? res_cols[dpiv[di]] : (size_t) -1;
				uint32_t *Ri = R + out * ldr;
				memset (Ri, 0, n * 4);
				if (xc < dc) {
					Ri[xc] = 1;
					for (size_t c = 0; c < nrem; ++c) Ri[res_cols[rem[c]]] = B2[xi * nrem + c];
					++xi;
				} else {
					Ri[dc] = 1;
					for (size_t c = 0; c < nrem; ++c) Ri[res_cols[rem[c]]] = D2[di * nrem + c];
					++di;
				}
				++out;
			}
			for (; out < m; ++out)
				memset (R + out * ldr, 0, n * 4);
			free (B1); free (B2);
		}
		*out_rows = rows_out;
		free (rem); free (dpos); free (D1); free (D2);
	} else {
		size_t rows_out;
		if (only_D) {
			/* MatrixGrid4 (:507-600) is handed D in its D2 slot while
			 * subst_splicer carries only source-0/1 column blocks, so the
			 * reference writes no entry of D here: row i of the output is
			 * the unit vector at the i-th non-pivot column of X.  The
			 * restatement keeps that behaviour bit for bit. */
			rows_out = rd;
			for (size_t i = 0; i < rd; ++i) {
				uint32_t *Ri = R + i * ldr;
				memset (Ri, 0, n * 4);
				Ri[res_cols[i]] = 1;
			}
		} else {
			rows_out = m;
			size_t xi = 0, di = 0, out = 0;
			while (xi < npiv || di < rd) {
				size_t xc = xi < npiv ? piv_cols[xi] : (size_t) -1;
				size_t dc = di < rd ? res_cols[dpiv[di]] : (size_t) -1;
				uint32_t *Ri = R + out * ldr;
				memset (Ri, 0, n * 4);
				if (xc < dc) {
					Ri[xc] = 1;
					for (size_t c = 0; c < nres; ++c) Ri[res_cols[c]] = B[xi * nres + c];
					++xi;
				} else {
					for (size_t c = 0; c < nres; ++c) Ri[res_cols[c]] = D[di * nres + c];
					++di;
				}
				++out;
			}
			for (; out < m; ++out)
				memset (R + out * ldr, 0, n * 4);
		}
		*out_rows = rows_out;
	}
	free (dpiv); free (is_dpiv);
out:
	free (A); free (B); free (C); free (D);
	free (piv_rows); free (res_rows); free (piv_cols); free (res_cols); free (col_pos);
	free (is_piv_row); free (is_piv_col);
	if (status == 2 && bad_row) *bad_row = bad;
	return status;
}

/* --------------------------------------------------------------- GF(2) -- */

static int getbit (const uint64_t *row, size_t j) { return (int) ((row[j >> 6] >> (j & 63)) & 1); }

/* GF(2) gemm as the generic Row x Row x Row path computes it without M4RI
 * (lela/blas/level3-generic.tcc:243-263 -> _gemv<GF2>, lela/blas/
 * level2-gf2.tcc:132-155 -> word XOR axpy, lela/blas/level1-gf2.tcc:
 * 281-298): row i of C is b*C_i XOR a*(XOR of the rows of B selected by
 * the set bits of row i of A). */
int oracle_gemm_gf2 (size_t m, size_t n, size_t k, int a,
		     const uint64_t *A, size_t lda, const uint64_t *B, size_t ldb,
		     int b, uint64_t *C, size_t ldc)
{
	size_t words = (n + 63) / 64;
	uint64_t tail = (n & 63) ? ((~0ULL) >> (64 - (n & 63))) : ~0ULL;
	for (size_t i = 0; i < m; ++i) {
		uint64_t *Ci = C + i * ldc;
		if (!b)
			memset (Ci, 0, words * 8);
		if (a)
			for (size_t l = 0; l < k; ++l)
				if (getbit (A + i * lda, l))
					for (size_t w = 0; w < words; ++w)
						Ci[w] ^= B[l * ldb + w];
		if (words)
			Ci[words - 1] &= tail;
	}
	return 0;
}

/* GF(2) non-reduced echelon form: the classical elimination of
 * oracle_echelon_zp_u32 with word-XOR row operations (the pivot is always
 * 1, so the multiplier of each eliminated row is 1). */
int oracle_echelon_gf2 (size_t m, size_t n, uint64_t *A, size_t lda, size_t *rank)
{
	size_t words = (n + 63) / 64;
	size_t i = 0, col = 0;
	uint64_t *tmp = (uint64_t *) malloc ((words ? words : 1) * 8);
	for (; i < m && col < n; ++i, ++col) {
		size_t prow = m;
		for (; col < n; ++col) {
			for (size_t r = i; r < m; ++r)
				if (getbit (A + r * lda, col)) { prow = r; break; }
			if (prow < m) break;
		}
		if (prow == m) break;
		if (prow != i) {
			memcpy (tmp, A + i * lda, words * 8);
			memcpy (A + i * lda, A + prow * lda, words * 8);
			memcpy (A + prow * lda, tmp, words * 8);
		}
		for (size_t r = i + 1; r < m; ++r)
			if (getbit (A + r * lda, col))
				for (size_t w = col >> 6; w < words; ++w)
					A[r * lda + w] ^= A[i * lda + w];
	}
	free (tmp);
	*rank = i;
	return 0;
}
