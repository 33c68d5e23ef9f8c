/* include/lela_cuda.h -- C ABI of the B200 (sm_100a) implementation of
 * LELA's exact linear-algebra hot path.
 *
 * Plain C: pointers, sizes and an int status.  No CUDA or C++ types appear
 * in the signatures, so the functions can be bound from C, C++ (the
 * CUDAModule in include/lela_cuda/cuda-module.h), ctypes or any FFI.
 *
 * Conventions
 *  - Matrices are row-major with an explicit leading dimension (row stride)
 *    counted in elements (uint32 for Z/p, 64-bit words for GF(2)); this is
 *    the `&A[0][0]` + `A.disp ()` view of a LELA DenseMatrix
 *    (lela/matrix/dense.h:319, 434) and of its submatrices (:425-429).
 *  - Z/p entries are canonical representatives in [0, p), p in [2, 2^32):
 *    the element convention of Modular<uint32> (lela/ring/modular.h:203-245).
 *  - GF(2) rows are packed LittleEndian: bit j of word w is column 64w + j,
 *    as LELA's BitVector<LittleEndian<uint64>> stores a DenseMatrix<bool>
 *    row (lela/vector/bit-iterator.h:249-296).
 *  - Functions without the _dev suffix take HOST pointers: the library
 *    copies inputs to the device, computes, copies results back and
 *    synchronises before returning.  The caller keeps ownership.
 *  - _dev functions take DEVICE pointers (on the handle's device) and are
 *    asynchronous on the handle's stream; device-side errors of an _dev call
 *    are reported by the next lela_cuda_synchronize().
 *  - A handle is not re-entrant (like a LELA Context, lela/blas/context.h:
 *    61-63): use one handle per host thread.
 *
 * Status codes map onto LELA's exceptions in the C++ layer:
 *  LELA_CUDA_DIAG_NOT_INVERTIBLE  -> DiagonalEntryNotInvertible(idx)
 *                                    (lela/util/error.h; thrown at
 *                                    lela/blas/level3-generic.tcc:441-442)
 *  LELA_CUDA_WRONG_MATRIX_FORM    -> WrongMatrixForm(row)
 *                                    (lela/algorithms/faugere-lachartre.tcc:32-41)
 *  LELA_CUDA_PIVOT_NOT_INVERTIBLE -> LELAError("Could not invert pivot-element
 *                                    in the ring") (lela/algorithms/elimination.tcc:106)
 *  LELA_CUDA_ERR_ARG              -> PreconditionFailed (lela_check, lela/util/debug.h)
 */
#ifndef LELA_CUDA_H
#define LELA_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct lela_cuda_ctx lela_cuda_ctx;

enum {
	LELA_CUDA_OK = 0,
	LELA_CUDA_ERR_ARG = 1,
	LELA_CUDA_ERR_CUDA = 2,
	LELA_CUDA_ERR_NOMEM = 3,
	LELA_CUDA_DIAG_NOT_INVERTIBLE = 4,
	LELA_CUDA_WRONG_MATRIX_FORM = 5,
	LELA_CUDA_PIVOT_NOT_INVERTIBLE = 6,
	LELA_CUDA_ERR_TIMEOUT = 7,
	LELA_CUDA_ERR_UNSUPPORTED = 8,
	LELA_CUDA_ERR_CAPACITY = 9  /* an output array is too small; see the call */
};

/* Kernel choice for the Z/p gemm (lela_cuda_set_gemm_kernel). */
enum {
	LELA_CUDA_GEMM_AUTO = 0,   /* small-K CUDA-core kernel for small problems, else tensor cores */
	LELA_CUDA_GEMM_PLAIN = 1,  /* CUDA-core delayed-reduction kernel */
	LELA_CUDA_GEMM_TC = 2,     /* limb-split INT8 tcgen05 kernel */
	LELA_CUDA_GEMM_SMALLK = 3  /* CUDA-core kernel for small K (unchecked sums when p < 2^28) */
};

/* ---------------------------------------------------------------- handle
 * Replaces the state a LELA Modules object owns (ZpModule's _tmp scratch,
 * lela/ring/modular.h:576; StrassenModule's sw, lela/algorithms/
 * strassen-winograd.h:148): stream, device workspace, kernel choice. */
int lela_cuda_create (lela_cuda_ctx **ctx, int device);
int lela_cuda_destroy (lela_cuda_ctx *ctx);
/* Use the caller's cudaStream_t (passed as void*); NULL restores the
 * handle's own stream. */
int lela_cuda_set_stream (lela_cuda_ctx *ctx, void *stream);
void *lela_cuda_get_stream (lela_cuda_ctx *ctx);
/* Wait for all work queued on the handle's stream and report any error a
 * kernel recorded (e.g. LELA_CUDA_ERR_TIMEOUT). */
int lela_cuda_synchronize (lela_cuda_ctx *ctx);
int lela_cuda_set_gemm_kernel (lela_cuda_ctx *ctx, int kernel);
/* Tile variant of the tensor-core Z/p gemm: 0 = automatic (variant 0 for
 * two limbs at k >= 512 and for four limbs, else variant 1), 1 = variant 0 (wide tiles: 256 / 128 / 32
 * columns for 1 / 2 / 4 limbs), 2 = variant 1 (128 / 64 columns for 1 / 2
 * limbs with two TMEM accumulator buffers, so the epilogue of one tile
 * overlaps the products of the next; four limbs always use variant 0).
 * For one limb the number of epilogue warps is chosen by k.
 * Every variant gives the same result.  No counterpart in the reference
 * (a tuning knob of the GPU kernels). */
int lela_cuda_set_gemm_tile (lela_cuda_ctx *ctx, int tile);
const char *lela_cuda_status_string (int status);
const char *lela_cuda_last_error (lela_cuda_ctx *ctx);
/* Number of SMs of the handle's device. */
int lela_cuda_num_sms (lela_cuda_ctx *ctx);
/* Kernel launches issued through the handle so far (all kernels). */
uint64_t lela_cuda_launch_count (lela_cuda_ctx *ctx);
/* Per-kernel device timing: when enabled, each launch of a main kernel
 * ("zp_gemm_tc", "zp_gemm_plain", ...) is bracketed by CUDA events on the
 * handle's stream; profile_read synchronises, returns the summed
 * milliseconds and launch count of one kernel name and forgets them. */
int lela_cuda_profile_enable (lela_cuda_ctx *ctx, int on);
int lela_cuda_profile_read (lela_cuda_ctx *ctx, const char *kernel, double *total_ms,
			    uint64_t *launches);
int lela_cuda_profile_reset (lela_cuda_ctx *ctx);

/* ------------------------------------------------------------- Z/p gemm
 * C <- a*A*B + b*C mod p, A m x k, B k x n, C m x n.
 * Replaces BLAS3::gemm (lela/blas/level3.h:82) for Modular<uint32> and dense
 * operands: _gemm<Modular<uint32>, Tag> reached through StrassenModule ->
 * ZpModule -> GenericModule (lela/blas/level3-sw.h:25-62,
 * lela/blas/level3-generic.tcc:285-322).
 * The host-pointer form returns when C holds the result.  For tensor-core
 * products with k <= 32768 and m >= 1024 it works in row blocks: B is
 * copied first, then A's and C's rows block by block on a second stream of
 * the handle, and each block's rows of C are copied back on a third while
 * later blocks still arrive.  Page-locked host buffers let the copies
 * overlap. */
int lela_cuda_gemm_zp_u32 (lela_cuda_ctx *ctx, size_t m, size_t n, size_t k, uint32_t p,
			   uint32_t a, const uint32_t *A, size_t lda, const uint32_t *B, size_t ldb,
			   uint32_t b, uint32_t *C, size_t ldc);
int lela_cuda_gemm_zp_u32_dev (lela_cuda_ctx *ctx, size_t m, size_t n, size_t k, uint32_t p,
			       uint32_t a, const uint32_t *A, size_t lda, const uint32_t *B,
			       size_t ldb, uint32_t b, uint32_t *C, size_t ldc);

/* ------------------------------------------------------------- Z/p trsm
 * B <- a * A^-1 * B, A m x m upper (upper != 0) or lower triangular, unit
 * diagonal when diag_is_one != 0, B m x n.
 * Replaces BLAS3::trsm (lela/blas/level3.h:121) ->
 * _trsm<Ring, GenericModule::Tag>::trsm_impl (lela/blas/level3-generic.tcc:
 * 421-498) for dense operands.  Returns LELA_CUDA_DIAG_NOT_INVERTIBLE with
 * *bad_idx = the index LELA's DiagonalEntryNotInvertible carries (smallest
 * singular index for lower, largest for upper); B is then unchanged.
 * With a = 0 the result is B = 0 and A is not inspected, as in LELA.
 * The _dev form synchronises the stream once (diagonal check). */
int lela_cuda_trsm_zp_u32 (lela_cuda_ctx *ctx, int upper, int diag_is_one, size_t m, size_t n,
			   uint32_t p, uint32_t a, const uint32_t *A, size_t lda, uint32_t *B,
			   size_t ldb, size_t *bad_idx);
int lela_cuda_trsm_zp_u32_dev (lela_cuda_ctx *ctx, int upper, int diag_is_one, size_t m,
			       size_t n, uint32_t p, uint32_t a, const uint32_t *A, size_t lda,
			       uint32_t *B, size_t ldb, size_t *bad_idx);
/* ------------------------------------- other Modular<T> element types
 * The Z/p gemm and trsm for matrices of Modular<uint8>, Modular<uint16>,
 * Modular<float> and Modular<double> elements (and Modular<uint32>, which
 * forwards to the _u32 entry points above).  elem is one of
 * LELA_CUDA_ELEM_*; A, B, C point to elements of that type, leading
 * dimensions count elements.  Element representation as in the reference
 * (lela/ring/modular.h:115-330): uint8 / uint16 hold 0 .. p-1; float /
 * double hold the symmetric representative -p/2 .. p/2 (integral values).
 * The scalars a, b are residues 0 .. p-1.  Moduli as the reference's
 * ModularTraits<T>::valid_modulus: p < 2^8, 2^16, 4096 (float), 2^26
 * (double); others return LELA_CUDA_ERR_ARG.  The results equal the
 * reference's BLAS3::gemm / BLAS3::trsm on Context<Modular<T>> (its float
 * and double gemm, lela/blas/level3-modular.tcc:25-122, is exact Z/p
 * arithmetic); for an even p the residue p/2 is stored as +p/2 (the
 * reference can give either sign).  Errors as for the _u32 forms. */
enum lela_cuda_elem {
	LELA_CUDA_ELEM_U8 = 1,
	LELA_CUDA_ELEM_U16 = 2,
	LELA_CUDA_ELEM_U32 = 4,
	LELA_CUDA_ELEM_F32 = 5,
	LELA_CUDA_ELEM_F64 = 6
};
int lela_cuda_gemm_zp (lela_cuda_ctx *ctx, int elem, size_t m, size_t n, size_t k, uint32_t p,
		       uint32_t a, const void *A, size_t lda, const void *B, size_t ldb, uint32_t b,
		       void *C, size_t ldc);
int lela_cuda_gemm_zp_dev (lela_cuda_ctx *ctx, int elem, size_t m, size_t n, size_t k, uint32_t p,
			   uint32_t a, const void *A, size_t lda, const void *B, size_t ldb,
			   uint32_t b, void *C, size_t ldc);
int lela_cuda_trsm_zp (lela_cuda_ctx *ctx, int elem, int upper, int diag_is_one, size_t m,
		       size_t n, uint32_t p, uint32_t a, const void *A, size_t lda, void *B,
		       size_t ldb, size_t *bad_idx);
int lela_cuda_trsm_zp_dev (lela_cuda_ctx *ctx, int elem, int upper, int diag_is_one, size_t m,
			   size_t n, uint32_t p, uint32_t a, const void *A, size_t lda, void *B,
			   size_t ldb, size_t *bad_idx);

/* The same solve with a sparse upper-triangular A (n x n) in CSR form:
 * row r's entries are colidx/vals[rowptr[r] .. rowptr[r+1]), rowptr[0] = 0;
 * B is n x ncols dense.  Replaces BLAS3::trsm on a SparseMatrix<uint32>
 * operand, e.g. FaugereLachartre's A^-1 B (lela/algorithms/
 * faugere-lachartre.tcc:791, UpperTriangular, diagIsOne = false), which
 * runs _trsm<Ring, GenericModule::Tag>::trsm_impl (lela/blas/
 * level3-generic.tcc:421-498) on the sparse rows.  Entries left of the
 * diagonal are ignored (an upper solve never reads them); a missing
 * diagonal entry is zero, reported like any singular diagonal
 * (LELA_CUDA_DIAG_NOT_INVERTIBLE, largest such index).  A column index >= n
 * returns LELA_CUDA_ERR_ARG.  A is expanded into a dense n x n device
 * scratch copy (4 n^2 bytes).  The _dev form takes device arrays. */
int lela_cuda_trsm_csr_upper_zp_u32 (lela_cuda_ctx *ctx, size_t n, size_t ncols, uint32_t p,
				     uint32_t a, int diag_is_one, const uint64_t *rowptr,
				     const uint32_t *colidx, const uint32_t *vals, uint32_t *B,
				     size_t ldb, size_t *bad_idx);
int lela_cuda_trsm_csr_upper_zp_u32_dev (lela_cuda_ctx *ctx, size_t n, size_t ncols, uint32_t p,
					 uint32_t a, int diag_is_one, const uint64_t *rowptr,
					 const uint32_t *colidx, const uint32_t *vals, uint32_t *B,
					 size_t ldb, size_t *bad_idx);
/* Diagonal-block solver of the trsm (and of the trsm steps inside
 * Faugere-Lachartre); every choice gives the same B. */
enum {
	LELA_CUDA_TRSM_AUTO = 0,    /* inverse leaves when B is wide, else block substitution */
	LELA_CUDA_TRSM_BLOCKS = 1,  /* 256-row blocks by substitution on CUDA cores */
	LELA_CUDA_TRSM_INVERSE = 2  /* 512-row blocks inverted, applied by the tensor-core gemm */
};
int lela_cuda_set_trsm_kernel (lela_cuda_ctx *ctx, int kernel);

/* ------------------------------------------------------- Z/p echelon form
 * A (m x n) <- its non-reduced row-echelon form, in place; *rank, *det =
 * product of the pivots.  Replaces EchelonForm::echelonize on a DenseMatrix
 * (lela/solutions/echelon-form.h:103-134: GaussJordan::echelonize +
 * Elimination::move_L), whose result equals Elimination::echelonize
 * (lela/algorithms/elimination.tcc:47-139) with DensePivotStrategy
 * (lela/algorithms/pivot-strategy.tcc:19-42): first nonzero in the column
 * at or below the current row, row transpositions, pivots not normalised.
 * LELA_CUDA_PIVOT_NOT_INVERTIBLE when Modular<uint32> cannot invert a pivot
 * (p >= 2^31). */
int lela_cuda_echelon_zp_u32 (lela_cuda_ctx *ctx, size_t m, size_t n, uint32_t p, uint32_t *A,
			      size_t lda, size_t *rank, uint32_t *det);
int lela_cuda_echelon_zp_u32_dev (lela_cuda_ctx *ctx, size_t m, size_t n, uint32_t p,
				  uint32_t *A, size_t lda, size_t *rank, uint32_t *det);

/* A (m x n) <- its reduced row-echelon form, in place: zero above and below
 * every pivot, zero rows last; *rank and *det as above.
 * unit_pivots = 0: the pivots keep their values, as EchelonForm::echelonize
 * (A, true) leaves a DenseMatrix with its default method (lela/solutions/
 * echelon-form.h:115-123: GaussJordan::echelonize_reduced, lela/algorithms/
 * gauss-jordan.tcc:434-466, through GaussJordanTransform, :27-230), whose
 * pivot rows are those of the non-reduced form with the later pivot columns
 * cleared.  unit_pivots = 1: every pivot row divided by its pivot, as the
 * standard method leaves it (echelon-form.h:108-111: Elimination::
 * echelonize_reduced, lela/algorithms/elimination.tcc:143-265).
 * LELA_CUDA_PIVOT_NOT_INVERTIBLE as above. */
int lela_cuda_echelon_reduced_zp_u32 (lela_cuda_ctx *ctx, size_t m, size_t n, uint32_t p,
				      uint32_t *A, size_t lda, int unit_pivots, size_t *rank,
				      uint32_t *det);
int lela_cuda_echelon_reduced_zp_u32_dev (lela_cuda_ctx *ctx, size_t m, size_t n, uint32_t p,
					  uint32_t *A, size_t lda, int unit_pivots, size_t *rank,
					  uint32_t *det);

/* PLUQ decomposition of the m x n matrix A in place: replaces
 * Elimination::pluq (lela/algorithms/elimination.h:196-209,
 * elimination.tcc:266-370) with DensePivotStrategy.  On return A holds U on
 * and above the diagonal (its columns in Q's order) and the multipliers of
 * L below it, as the reference leaves them; P and Q receive the row and
 * column transpositions as pairs (P[2t], P[2t+1]) in the reference's order
 * (reversed, elimination.tcc:362-363), *np / *nq pairs each (room for
 * min(m, n) pairs); *rank and *det = product of the pivots.
 * LELA_CUDA_PIVOT_NOT_INVERTIBLE when a pivot cannot be inverted (A then
 * unspecified).  The _dev form takes A on the device (P, Q on the host). */
int lela_cuda_pluq_zp_u32 (lela_cuda_ctx *ctx, size_t m, size_t n, uint32_t p, uint32_t *A,
			   size_t lda, size_t *P, size_t *np, size_t *Q, size_t *nq, size_t *rank,
			   uint32_t *det);
int lela_cuda_pluq_zp_u32_dev (lela_cuda_ctx *ctx, size_t m, size_t n, uint32_t p, uint32_t *A,
			       size_t lda, size_t *P, size_t *np, size_t *Q, size_t *nq,
			       size_t *rank, uint32_t *det);

/* The standard method's reduced row-echelon form together with its
 * transform: replaces Elimination::echelonize_reduced (A, L, P, rank, det,
 * compute_L = true) (lela/algorithms/elimination.h:108-162,
 * elimination.tcc:143-265) with DensePivotStrategy.  On return A (m x n)
 * holds the reduced form with unit pivots (as lela_cuda_echelon_reduced_
 * zp_u32 with unit_pivots = 1), L (m x m, row stride ldl >= m) the matrix
 * with A_out = L P A_in, where P applies the row transpositions
 * (P[2t], P[2t+1]), t < *np, in that order (the reference's order, not
 * reversed; room for min(m, n) pairs).  L is [[X, 0], [Y, I]] in blocks of
 * *rank rows and columns.  *det = product of the pivots before scaling.
 * p must be below 2^31 (LELA_CUDA_ERR_ARG otherwise): above it
 * Modular<uint32>::inv works in wrapped 32-bit ints and returns no true
 * inverse, so the reference itself produces no transform.
 * LELA_CUDA_PIVOT_NOT_INVERTIBLE when a pivot cannot be inverted (a
 * composite p; A and L unspecified).  The _dev form takes A and L on the
 * device (P on the host). */
int lela_cuda_echelon_reduced_transform_zp_u32 (lela_cuda_ctx *ctx, size_t m, size_t n,
						uint32_t p, uint32_t *A, size_t lda, uint32_t *L,
						size_t ldl, size_t *P, size_t *np, size_t *rank,
						uint32_t *det);
int lela_cuda_echelon_reduced_transform_zp_u32_dev (lela_cuda_ctx *ctx, size_t m, size_t n,
						    uint32_t p, uint32_t *A, size_t lda, uint32_t *L,
						    size_t ldl, size_t *P, size_t *np, size_t *rank,
						    uint32_t *det);

/* ------------------------------------------- Faugere-Lachartre echelon form
 * Echelon form of the F4 matrix X (m x n, CSR: rowptr[m+1], colidx, vals;
 * column indices strictly increasing within a row, stored values in [0,p)).
 * Replaces FaugereLachartre<Modular<uint32>>::echelonize (lela/algorithms/
 * faugere-lachartre.h:80-81, .tcc:735-917) with R returned dense (row stride
 * ldr >= n): reduced != 0 gives the reduced row-echelon form (m rows, zero
 * rows last); only_D as in the reference (*out_rows = rank of D rows).
 * *rank and *det are the reference's outputs (det = product of the leading
 * entries of the X pivot rows and of the echelon form of D).
 * Status: LELA_CUDA_WRONG_MATRIX_FORM with *bad_row (rows not sorted by
 * leading column: WrongMatrixForm, faugere-lachartre.tcc:80-81);
 * LELA_CUDA_DIAG_NOT_INVERTIBLE when A's diagonal cannot be inverted (the
 * reference returns early from echelonize, :792-799; R is then untouched).
 * The _dev form takes the CSR arrays and R on the device. */
int lela_cuda_fl_echelonize_zp_u32 (lela_cuda_ctx *ctx, size_t m, size_t n, uint32_t p,
				    const uint64_t *rowptr, const uint32_t *colidx,
				    const uint32_t *vals, int reduced, int only_D, uint32_t *R,
				    size_t ldr, size_t *rank, uint32_t *det, size_t *out_rows,
				    size_t *bad_row);
int lela_cuda_fl_echelonize_zp_u32_dev (lela_cuda_ctx *ctx, size_t m, size_t n, uint32_t p,
					const uint64_t *rowptr, const uint32_t *colidx,
					const uint32_t *vals, int reduced, int only_D, uint32_t *R,
					size_t ldr, size_t *rank, uint32_t *det, size_t *out_rows,
					size_t *bad_row);
/* The same, with R returned as CSR rows -- the SparseMatrix<uint32> the
 * reference writes (faugere-lachartre.tcc:860-911): R_rowptr[*out_rows + 1]
 * (room for m + 1 entries), R_colidx / R_vals with room for R_cap entries,
 * column indices strictly increasing within a row.  No dense m x n array
 * is formed (at m = 120000 that would be 69 GB).  *R_nnz = the result's
 * entries.  When R_cap < *R_nnz the call writes R_rowptr, returns
 * LELA_CUDA_ERR_CAPACITY and keeps the result in the handle until its next
 * Faugere-Lachartre call: lela_cuda_fl_csr_fetch copies the entries out
 * then.  Other statuses as above.  _csr takes host arrays, _csr_dev device
 * arrays (asynchronous apart from one synchronisation that sizes the
 * result). */
int lela_cuda_fl_echelonize_zp_u32_csr (lela_cuda_ctx *ctx, size_t m, size_t n, uint32_t p,
					const uint64_t *rowptr, const uint32_t *colidx,
					const uint32_t *vals, int reduced, int only_D,
					uint64_t *R_rowptr, uint32_t *R_colidx, uint32_t *R_vals,
					size_t R_cap, size_t *R_nnz, size_t *rank, uint32_t *det,
					size_t *out_rows, size_t *bad_row);
int lela_cuda_fl_echelonize_zp_u32_csr_dev (lela_cuda_ctx *ctx, size_t m, size_t n, uint32_t p,
					    const uint64_t *rowptr, const uint32_t *colidx,
					    const uint32_t *vals, int reduced, int only_D,
					    uint64_t *R_rowptr, uint32_t *R_colidx, uint32_t *R_vals,
					    size_t R_cap, size_t *R_nnz, size_t *rank, uint32_t *det,
					    size_t *out_rows, size_t *bad_row);
/* Copies the kept CSR result's column indices and values (cap >= its entry
 * count) into host (device = 0) or device (device != 0) arrays.  No
 * counterpart in the reference. */
int lela_cuda_fl_csr_fetch (lela_cuda_ctx *ctx, uint32_t *colidx, uint32_t *vals, size_t cap,
			    int device);

/* ----------------------------------------------------------------- GF(2)
 * Packed rows (bit j of 64-bit word w = column 64w + j), strides in words.
 * C <- a*A*B + b*C with a, b in {0, 1}.  Replaces BLAS3::gemm over GF2 on
 * DenseMatrix<bool>: without M4RI the generic Row*Row*Row gemm
 * (lela/blas/level3-generic.tcc:243-263 -> lela/blas/level2-gf2.tcc:132-155),
 * with M4RI mzd_mul/mzd_addmul (lela/blas/level3-m4ri.tcc:78-80).
 * Kernels (lela_cuda_set_gf2_kernel): 0 = auto (tensor cores), 1 =
 * int8-expanded tcgen05, 2 = bit-packed four-Russians on CUDA cores.
 * When n is not a multiple of 64, the bits of each row's last word of C at
 * columns >= n are left as they were (a strided view may keep the next
 * columns of a wider matrix there). */
int lela_cuda_set_gf2_kernel (lela_cuda_ctx *ctx, int kernel);
int lela_cuda_gemm_gf2 (lela_cuda_ctx *ctx, size_t m, size_t n, size_t k, int a,
			const uint64_t *A, size_t lda, const uint64_t *B, size_t ldb, int b,
			uint64_t *C, size_t ldc);
int lela_cuda_gemm_gf2_dev (lela_cuda_ctx *ctx, size_t m, size_t n, size_t k, int a,
			    const uint64_t *A, size_t lda, const uint64_t *B, size_t ldb, int b,
			    uint64_t *C, size_t ldc);
/* A (m x n) <- its non-reduced row-echelon form over GF(2), in place; *rank.
 * Replaces EchelonForm<GF2>::echelonize on a DenseMatrix<bool> without M4RI
 * (GaussJordan + move_L, lela/solutions/echelon-form.h:103-134), equal to
 * Elimination::echelonize with the dense pivot rule (first row with a 1,
 * transpositions; lela/algorithms/pivot-strategy.tcc:44-66). */
int lela_cuda_echelon_gf2 (lela_cuda_ctx *ctx, size_t m, size_t n, uint64_t *A, size_t lda,
			   size_t *rank);
int lela_cuda_echelon_gf2_dev (lela_cuda_ctx *ctx, size_t m, size_t n, uint64_t *A, size_t lda,
			       size_t *rank);

/* --------------------------------------------------------------- batches
 * No single LELA counterpart: these run many independent instances of the
 * routines above (EchelonForm::echelonize on dense blocks, FaugereLachartre
 * ::echelonize) per call, with the same results per instance.
 *
 * Dense Z/p echelon blocks, all matrices on the DEVICE, descriptors on the
 * host.  kernel[i] (or NULL = all 0): 0 = automatic (blocks that fit one
 * CTA's shared memory go to the batched kernel, the rest to the panel
 * pipeline with tensor-core updates), 1 = batched shared-memory kernel,
 * 2 = panel pipeline with tensor-core updates (wide tiles), 3 = panel
 * pipeline with CUDA-core updates, 4 = panel pipeline with tensor-core
 * updates on tiles with two accumulator buffers (see
 * lela_cuda_set_gemm_tile).  The shared-memory blocks are processed by one
 * persistent launch captured in a CUDA graph (the instantiated graph is kept
 * in the handle and replayed while the count of such blocks stays the same);
 * when two or more blocks take the panel pipeline they are spread over up to
 * 8 worker handles with their own streams, concurrently with that launch, so
 * the call first waits for the work already queued on the handle's stream.
 * status[i] = 0 or LELA_CUDA_PIVOT_NOT_INVERTIBLE. */
int lela_cuda_echelon_zp_u32_batch (lela_cuda_ctx *ctx, size_t count, uint32_t *const *A,
				    const size_t *lda, const size_t *m, const size_t *n,
				    const uint32_t *p, const int *kernel, size_t *rank,
				    uint32_t *det, int *status);
/* Faugere-Lachartre on `count` CSR matrices (arrays on the DEVICE; R[i] is a
 * device output of m[i] rows, stride ldr[i]), spread over nworkers threads
 * with their own streams, largest first.  status[i] as for the single call.
 * Memory-budgeted queue: when the nworkers largest matrices may not fit in
 * the budget together (estimate per matrix: 4 m n + 4 (m + n) m + 2 KB per
 * row + 256 MB), a matrix starts only when its estimate fits beside those
 * running (one that does not fit even alone runs alone), and each worker
 * frees its device buffers after a matrix.  The batch is stream-ordered on
 * the handle's stream: the workers start after the work queued there, and
 * work queued there after the call starts after the batch. */
/* Budget of that queue in bytes; 0 (the default) = 90 % of the free device
 * memory at the call plus what the worker handles already hold. */
int lela_cuda_set_batch_memory_budget (lela_cuda_ctx *ctx, size_t bytes);
int lela_cuda_fl_echelonize_zp_u32_batch (lela_cuda_ctx *ctx, size_t count, const size_t *m,
					  const size_t *n, const uint32_t *p,
					  const uint64_t *const *rowptr, const uint32_t *const *colidx,
					  const uint32_t *const *vals, uint32_t *const *R,
					  const size_t *ldr, int reduced, int nworkers, size_t *rank,
					  uint32_t *det, int *status);

/* ------------------------------------------------------------ cost model
 * No reference counterpart (LELA chooses implementations at compile time).
 * A fully connected FP32 network nfeat -> 64 -> 64 -> 1 with ReLU that
 * predicts the log time of a kernel choice from block features; its choice
 * never changes a result.  All pointers are DEVICE pointers; parameters are
 * one float array laid out W1[nfeat][64], b1[64], W2[64][64], b2[64],
 * W3[64], b3 (lela_cuda_mlp_param_count floats), nfeat <= 16.
 * mlp_grad zeroes grad and loss, then writes d(MSE)/d(params) and the MSE;
 * mlp_adam applies one Adam step (step counts from 1). */
size_t lela_cuda_mlp_param_count (int nfeat);
int lela_cuda_mlp_forward (lela_cuda_ctx *ctx, const float *params, int nfeat, const float *X,
			   size_t n, float *out);
int lela_cuda_mlp_grad (lela_cuda_ctx *ctx, const float *params, int nfeat, const float *X,
			const float *target, size_t n, float *grad, float *loss);
int lela_cuda_mlp_adam (lela_cuda_ctx *ctx, float *params, const float *grad, float *m, float *v,
			size_t count, int step, float lr);

/* The same tensor-core gemm for callers that cannot allocate device memory:
 * code whose device memory is owned by someone else (a host framework's
 * caching allocator, a fixed per-process budget) or that must not call
 * cudaMalloc/cudaFree because they may synchronise the device.  No
 * counterpart in the reference: LELA has no device code.
 *
 * A, B and C are DEVICE pointers on the current device; `stream` is a
 * cudaStream_t (NULL = legacy default stream).  No handle is needed and
 * nothing is allocated: the kernel's scratch (the 8-bit limb planes of A and
 * B) lives in a fixed 64 MiB __device__ array inside the library, which
 * every GPU that loads the library keeps until the process exits.
 *  - Limit: L*(m+n)*round16(min(k,32768)) <= 64 MiB, with L = 1, 2 or 4
 *    limbs for p <= 2^8, 2^16, 2^32 (m = n = k = 4096 fits at p = 65521);
 *    larger problems return LELA_CUDA_ERR_ARG before any GPU work.
 *  - The first call on a device sets up that device (looks up the array's
 *    device address); make it before any stream capture.  That set-up is
 *    kept for the life of the process: do not call this entry point after
 *    cudaDeviceReset, which invalidates the address it looked up.
 *  - All calls share the array and it keeps the last call's contents; calls
 *    whose GPU work overlaps (other streams or threads without ordering)
 *    race on it.  The call synchronises `stream` before returning. */
int lela_cuda_gemm_zp_u32_noalloc (size_t m, size_t n, size_t k, uint32_t p, uint32_t a,
				   const uint32_t *A, size_t lda, const uint32_t *B, size_t ldb,
				   uint32_t b, uint32_t *C, size_t ldc, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* LELA_CUDA_H */
