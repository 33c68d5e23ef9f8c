/* oracle/lela_oracle.h -- CPU restatement of LELA's exact linear-algebra
 * hot path, in plain C.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py load this library, and only as the checker.
 * The product (lela_b200/, include/) never calls it.
 *
 * Every function restates the reference routine cited beside it
 * (paths relative to the LELA source tree).  The restatement is itself
 * checked against LELA's own code (oracle/_ref/liblela_ref.so) and against
 * the committed fixtures in tests/golden/.
 *
 * Matrices are row-major with an explicit leading dimension (elements for
 * Z/p, 64-bit words for GF(2)).  GF(2) rows use LELA's LittleEndian packing:
 * bit j of word w is column 64*w + j.
 */
#ifndef LELA_ORACLE_H
#define LELA_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* C <- a*A*B + b*C mod p. */
int oracle_gemm_zp_u32 (uint32_t p, size_t m, size_t n, size_t k, uint32_t a,
			const uint32_t *A, size_t lda, const uint32_t *B, size_t ldb,
			uint32_t b, uint32_t *C, size_t ldc);

/* Same, rows of C split over nthreads POSIX threads. */
int oracle_gemm_zp_u32_threads (int nthreads, uint32_t p, size_t m, size_t n, size_t k, uint32_t a,
				const uint32_t *A, size_t lda, const uint32_t *B, size_t ldb,
				uint32_t b, uint32_t *C, size_t ldc);

/* B <- a*A^-1*B mod p, A m x m triangular.  Returns 0, or 1 and *bad_idx
 * for a diagonal entry that is not invertible. */
int oracle_trsm_zp_u32 (uint32_t p, int upper, int diag_is_one, size_t m, size_t n, uint32_t a,
			const uint32_t *A, size_t lda, uint32_t *B, size_t ldb, size_t *bad_idx);

/* Non-reduced row echelon form in place; rank and det = product of pivots.
 * Returns 0, or -1 when a pivot is not invertible mod p. */
int oracle_echelon_zp_u32 (uint32_t p, size_t m, size_t n, uint32_t *A, size_t lda,
			   size_t *rank, uint32_t *det);

/* Reduced row echelon form in place (pivots keep their values; zeros above
 * and below them); rank and det as above.  Returns 0, or -1 when a pivot is
 * not invertible mod p. */
int oracle_echelon_reduced_zp_u32 (uint32_t p, size_t m, size_t n, uint32_t *A, size_t lda,
				   size_t *rank, uint32_t *det);

/* The same with every pivot row divided by its pivot (pivots 1): the
 * standard method's reduced form. */
int oracle_echelon_reduced_unit_zp_u32 (uint32_t p, size_t m, size_t n, uint32_t *A, size_t lda,
					size_t *rank, uint32_t *det);

/* The standard method's reduced form (pivots 1) with its transform: A <- R,
 * L (m x m, ldl) <- the matrix with R = L P A_in, P the row transpositions
 * as pairs (at most min(m, n)) in the order they were applied.  Returns 0,
 * or -1 when a pivot is not invertible mod p. */
int oracle_echelon_reduced_L_zp_u32 (uint32_t p, size_t m, size_t n, uint32_t *A, size_t lda,
				     uint32_t *L, size_t ldl, size_t *P, size_t *np,
				     size_t *rank, uint32_t *det);

/* The fast method's reduced form (pivots keep their values) with its
 * transform: the same with every pivot row of A and L multiplied by its
 * pivot; R = L P A_in as above. */
int oracle_gj_echelon_reduced_L_zp_u32 (uint32_t p, size_t m, size_t n, uint32_t *A, size_t lda,
					uint32_t *L, size_t ldl, size_t *P, size_t *np,
					size_t *rank, uint32_t *det);

/* Non-reduced row echelon form with L kept below the diagonal: A <- U plus
 * the strictly lower part of the transform T (T P A_in = U); gj = 0 as
 * Elimination::echelonize (det = product of the pivots), gj = 1 as
 * GaussJordan::echelonize (the same A and P; det as GaussTransform computes
 * it).  P as pairs in the order applied.  Returns 0, or -1 when a pivot is
 * not invertible mod p. */
int oracle_echelon_packed_L_zp_u32 (int gj, uint32_t p, size_t m, size_t n, uint32_t *A,
				    size_t lda, size_t *P, size_t *np, size_t *rank, uint32_t *det);

/* PLUQ decomposition in place (L strictly below the diagonal, U on and
 * above it); P and Q as transposition pairs (at most min(m, n) each), in
 * the reference's order; rank, det = product of the pivots.  Returns 0, or
 * -1 when a pivot is not invertible mod p. */
int oracle_pluq_zp_u32 (uint32_t p, size_t m, size_t n, uint32_t *A, size_t lda,
			size_t *P, size_t *np, size_t *Q, size_t *nq, size_t *rank, uint32_t *det);

/* Faugere-Lachartre echelon form of a CSR matrix.  R is dense m x n (ldr).
 * Returns 0; 1 with *bad_row on a malformed input (WrongMatrixForm);
 * 2 when the pivot block is singular (the reference returns early). */
int oracle_fl_echelonize_zp_u32 (uint32_t p, size_t m, size_t n,
				 const uint64_t *rowptr, const uint32_t *colidx, const uint32_t *vals,
				 int reduced, int only_D,
				 uint32_t *R, size_t ldr, size_t *rank, uint32_t *det,
				 size_t *out_rows, size_t *bad_row);

/* GF(2): C <- a*A*B + b*C. */
int oracle_gemm_gf2 (size_t m, size_t n, size_t k, int a,
		     const uint64_t *A, size_t lda, const uint64_t *B, size_t ldb,
		     int b, uint64_t *C, size_t ldc);

/* GF(2) non-reduced row echelon form in place; returns rank in *rank. */
int oracle_echelon_gf2 (size_t m, size_t n, uint64_t *A, size_t lda, size_t *rank);

/* Scalar helpers used by the tests. */
uint32_t oracle_inv_zp (uint32_t p, uint32_t x);  /* 0 when not invertible */

#ifdef __cplusplus
}
#endif
#endif
