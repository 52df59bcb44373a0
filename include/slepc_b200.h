/*
 * slepc_b200.h -- C ABI of the B200-native Krylov-Schur inner loop.
 *
 * Plain C: opaque handles, plain pointers and sizes, an explicit CUDA stream
 * (passed as void*) and an int status.  Every entry point names the SLEPc
 * interface it replaces (paths relative to the SLEPc 3.22 source tree).
 *
 * Four object kinds mirror SLEPc's:
 *   b200_mat  -- a CSR matrix resident in HBM with a hand-written SpMV
 *                (the new Mat SpMV type, in place of MATAIJCUSPARSE's MatMult),
 *                or the cross-product shell A^T A of the SVD cross solver
 *   b200_bv   -- a column-major basis of vectors resident in HBM
 *                (the new BV type: the BVOps table of bvimpl.h:25-61)
 *   b200_eps  -- the Hermitian Krylov-Schur solver that drives them
 *                (EPSSolve with EPSKRYLOVSCHUR, problem type EPS_HEP)
 *   b200_svd  -- the SVD cross solver (SVDCROSS): Krylov-Schur on A^T A
 *
 * Pointers marked _dev are device (HBM) addresses; pointers marked _host are
 * host addresses.  All work is ordered on the object's stream; entry points
 * that return host values synchronise that stream.
 */
#ifndef SLEPC_B200_H
#define SLEPC_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes (the PetscErrorCode analogue; 0 = success). */
typedef int b200_status;
#define B200_OK 0
#define B200_ERR_ARG 1        /* invalid argument (PETSC_ERR_ARG_OUTOFRANGE / _SIZ / _WRONG) */
#define B200_ERR_CUDA 2       /* a CUDA runtime call failed */
#define B200_ERR_LAPACK 3     /* LAPACK returned info != 0 (SlepcCheckLapackInfo) */
#define B200_ERR_INNER 4      /* invalid inner product (BV_SafeSqrt, bvimpl.h:121-141) */
#define B200_ERR_BREAKDOWN 5  /* start vector zero or in the deflation space (epssolve.c:864-867) */
#define B200_ERR_NOMEM 6      /* device allocation failed */
#define B200_ERR_STATE 7      /* call out of order (e.g. EPSGetEigenpair before EPSSolve) */
#define B200_ERR_DEVICE 8     /* a kernel reported a device-side error (bounded wait expired, NaN) */
#define B200_ERR_FP 9         /* floating-point failure (PETSC_ERR_FP: negative eigenvalue of A^T A) */
#define B200_ERR_IO 10        /* file read/write failure or malformed binary file (PETSC_ERR_FILE_READ / _UNEXPECTED) */
#define B200_ERR_SUP 11       /* an option this implementation does not provide (PETSC_ERR_SUP) */

/* Which eigenpairs (EPSWhich, include/slepceps.h; comparators src/sys/slepcsc.c:152-210). */
#define B200_LARGEST_MAGNITUDE 1
#define B200_SMALLEST_MAGNITUDE 2
#define B200_LARGEST_REAL 3
#define B200_SMALLEST_REAL 4

/* Converged reasons (EPSConvergedReason, include/slepceps.h). */
#define B200_CONVERGED_TOL 1
#define B200_CONVERGED_ITERATING 0
#define B200_DIVERGED_ITS (-1)
#define B200_DIVERGED_BREAKDOWN (-2)

/* Error types for b200_eps_compute_error (EPSErrorType). */
#define B200_ERROR_ABSOLUTE 0
#define B200_ERROR_RELATIVE 1

/* Storage types of matrix values (PETSc's MatScalar: double, or single with
 * --with-precision=single).  Products and sums are FP64 for both. */
#define B200_SCALAR_F64 0
#define B200_SCALAR_F32 1

/* Which singular triplets (SVDWhich, include/slepcsvd.h). */
#define B200_SVD_LARGEST 0
#define B200_SVD_SMALLEST 1

/* Error type for b200_svd_compute_error in addition to ABSOLUTE/RELATIVE (SVD_ERROR_NORM). */
#define B200_ERROR_NORM 2

/* PETSc binary files (PetscViewerBinary): class ids of the objects and file modes. */
#define B200_MAT_FILE_CLASSID 1211216
#define B200_VEC_FILE_CLASSID 1211214
#define B200_FILE_MODE_READ 0
#define B200_FILE_MODE_WRITE 1
#define B200_FILE_MODE_APPEND 2
/* b200_mat_load storage: a square CSR operator (b200_mat_create_csr), else a scalar type of b200_mat_create_aij. */
#define B200_MAT_OPERATOR (-1)

typedef struct b200_viewer_s *b200_viewer;
typedef struct b200_mat_s *b200_mat;
typedef struct b200_bv_s *b200_bv;
typedef struct b200_eps_s *b200_eps;
typedef struct b200_svd_s *b200_svd;
typedef struct b200_batch_s *b200_batch;

/* Library information and the last error message (thread-local). */
const char *b200_version(void);
const char *b200_last_error(void);
/* Number of kernels this library has launched in this process (all devices). */
uint64_t b200_kernel_launch_count(void);

/* ------------------------------------------------------------------ Mat --- */

/* Create a square CSR matrix in HBM from host arrays (copied).  Replaces
 * MatCreateSeqAIJWithArrays + MatSetType(MATAIJCUSPARSE) + MatAssembly, whose
 * MatMult is called from BVMatMultColumn (src/sys/classes/bv/interface/bvops.c:862-890)
 * and STApply (src/sys/classes/st/interface/stsolve.c:45-60). */
b200_status b200_mat_create_csr(int n, int64_t nnz, const int *rowptr_host, const int *colind_host,
                                const double *vals_host, void *stream, b200_mat *A);
/* Same, from arrays already in HBM (copied device to device). */
b200_status b200_mat_create_csr_device(int n, int64_t nnz, const int *rowptr_dev, const int *colind_dev,
                                       const double *vals_dev, void *stream, b200_mat *A);
/* Create a general m x n CSR matrix from host arrays (copied), values stored
 * as B200_SCALAR_F64 (double *) or B200_SCALAR_F32 (float *).  The explicit
 * transpose is built on the host at creation and kept in HBM beside A, the
 * transpose SVDSetUp builds with MatHermitianTranspose
 * (src/svd/interface/svdsetup.c:300-314); rows of A longer than 256 nonzeros
 * (and of A^T: the power-law columns of A) are split into segments whose
 * partial sums are added in a fixed order. */
b200_status b200_mat_create_aij(int m, int n, int64_t nnz, const int *rowptr_host, const int *colind_host,
                                const void *vals_host, int scalar_type, void *stream, b200_mat *A);
/* The shell C = A^T A of SVDCROSS (MatMult_Cross, src/svd/impls/cross/cross.c:31-41):
 * y = A^T (A x) through a device work vector of length m.  A must be created by
 * b200_mat_create_aij and outlive C.  C is the EPS operator of the cross solver. */
b200_status b200_mat_create_cross(b200_mat A, b200_mat *C);
/* y = A x on device vectors (MatMult); for a cross shell y = A^T A x. */
b200_status b200_mat_mult(b200_mat A, const double *x_dev, double *y_dev);
/* y = A^T x (MatMultTranspose) for a matrix from b200_mat_create_aij. */
b200_status b200_mat_mult_transpose(b200_mat A, const double *x_dev, double *y_dev);
/* Number of columns (the operator dimension of a square or cross operator) and nonzeros. */
b200_status b200_mat_get_size(b200_mat A, int *n, int64_t *nnz);
/* MatGetSize: rows and columns. */
b200_status b200_mat_get_sizes(b200_mat A, int *m, int *n);
/* MatNorm(NORM_INFINITY), known for matrices created from host arrays. */
b200_status b200_mat_norm_inf(b200_mat A, double *nrm);
/* CSR SpMV schedule of a matrix (a MatSetOption-style knob):
 *   B200_SPMV_SELL (default)  -- sliced ELL, 32-row slices, one row per lane (rows <= 32 nonzeros;
 *                                longer rows by warp tiles and segments);
 *   B200_SPMV_WARPTILE        -- warp tiles of <= 32 rows / <= 256 nonzeros;
 *   B200_SPMV_PIPELINED       -- the warp tiles with the next tile's loads in flight;
 *   B200_SPMV_ROWBLOCK        -- CTA row blocks of <= 1024 rows / <= 4096 nonzeros (FP64 only).
 * All sum each row of at most 256 nonzeros in index order (the bits of a sequential loop). */
#define B200_SPMV_ROWBLOCK 0
#define B200_SPMV_WARPTILE 1
/* warp tiles with a two-tile software pipeline (next tile's loads in flight; same bits) */
#define B200_SPMV_PIPELINED 2
/* sliced ELL, 32-row slices, one row per lane, for rows of at most 32 nonzeros (longer rows:
 * warp tiles / segments); a second copy of the entries in HBM; same bits */
#define B200_SPMV_SELL 3
b200_status b200_mat_set_spmv_schedule(b200_mat A, int schedule);
/* Lanes per row chosen for the SpMV (1..32), for tests and reports. */
b200_status b200_mat_get_lanes(b200_mat A, int *lanes);
b200_status b200_mat_destroy(b200_mat A);

/* Stateless SpMV on raw device CSR arrays (the kernel behind b200_mat_mult). */
b200_status b200_csr_spmv(int n, const int *rowptr_dev, const int *colind_dev, const double *vals_dev,
                          const double *x_dev, double *y_dev, int lanes, void *stream);

/* ------------------------------------------------------------------- BV --- */

/* Create a basis of m columns of length n in HBM (BVCreate + BVSetSizes +
 * BVSetType, src/sys/classes/bv/interface/bvbasic.c).  Columns are stored
 * column-major with a leading dimension ld >= n (a multiple of 32). */
b200_status b200_bv_create(int n, int m, void *stream, b200_bv *bv);
b200_status b200_bv_destroy(b200_bv bv);
b200_status b200_bv_get_sizes(b200_bv bv, int *n, int *m, int *ld);
/* Device address of the storage (BVGetArray, bvimpl.h getarray). */
b200_status b200_bv_get_array(b200_bv bv, double **V_dev);
/* BVSetActiveColumns / BVGetActiveColumns (bvbasic.c). */
b200_status b200_bv_set_active_columns(b200_bv bv, int l, int k);
b200_status b200_bv_get_active_columns(b200_bv bv, int *l, int *k);
/* BVSetOrthogonalization eta (bvfunc.c:178 default 0.7071); CGS with refinement if needed. */
b200_status b200_bv_set_orthog_eta(b200_bv bv, double eta);
/* BVSetOrthogonalization / BVGetOrthogonalization block type (BVOrthogBlockType,
 * include/slepcbv.h:84-88; bvbasic.c:975-987; default GS, bvfunc.c:179): the
 * method of b200_bv_orthogonalize.  TSQR and TSQRCHOL (bvorthog.c:615-660) run
 * the Householder QR of the active columns on the device with one process's
 * semantics of bvlapack.c:347-560 (geqrf + orgqr; R with LAPACK's signs);
 * TSQRCHOL factors a copy and applies R^{-1}.  Both need n >= k - l. */
#define B200_ORTHOG_BLOCK_GS 0
#define B200_ORTHOG_BLOCK_CHOL 1
#define B200_ORTHOG_BLOCK_TSQR 2
#define B200_ORTHOG_BLOCK_TSQRCHOL 3
#define B200_ORTHOG_BLOCK_SVQB 4
b200_status b200_bv_set_orthog_block(b200_bv bv, int type);
b200_status b200_bv_get_orthog_block(b200_bv bv, int *type);
/* Copy a column from/to host memory (BVGetColumn + VecGetArray / VecSetValues). */
b200_status b200_bv_set_column(b200_bv bv, int j, const double *x_host);
b200_status b200_bv_get_column(b200_bv bv, int j, double *x_host);
/* Copy column j to/from a device vector (BVCopyVec / BVInsertVec). */
b200_status b200_bv_copy_vec(b200_bv bv, int j, double *x_dev);
b200_status b200_bv_insert_vec(b200_bv bv, int j, const double *x_dev);

/* BVOrthogonalizeColumn (src/sys/classes/bv/interface/bvorthog.c:315-340):
 * classical Gram-Schmidt against columns 0..j-1 with DGKS refinement "if
 * needed" (bvorthog.c:145-217).  H_host (nullable) receives j+1 values: the
 * coefficients and then the norm. */
b200_status b200_bv_orthogonalize_column(b200_bv bv, int j, double *H_host, double *norm, int *lindep);
/* BVOrthonormalizeColumn (bvorthog.c:380-427, replace = FALSE): the same,
 * then column j is scaled by 1/norm. */
b200_status b200_bv_orthonormalize_column(b200_bv bv, int j, double *norm, int *lindep);
/* BVOrthogonalizeVec (bvorthog.c:238-262): a device vector against the k active columns. */
b200_status b200_bv_orthogonalize_vec(b200_bv bv, double *v_dev, double *H_host, double *norm, int *lindep);
/* One classical Gram-Schmidt pass: the BV gramschmidt op
 * (include/slepc/private/bvimpl.h:53), which BVOrthogonalizeGS's DGKS loop
 * (src/sys/classes/bv/interface/bvorthog.c:174-203) calls 1-3 times in place
 * of BVOrthogonalizeCGS1 (bvorthog.c:91-132).  v_dev null: column j of the BV
 * against columns 0..j-1; otherwise the device vector v_dev against the k
 * active columns (j ignored).  c_dev (device, nullable, jb+1 entries with jb =
 * j or k) receives this pass's coefficients V^T w and, at position jb, w^T w;
 * h_dev (device, nullable) accumulates h += c over the jb coefficients
 * (BV_AddCoefficients) -- for the column variant a null h_dev accumulates
 * into the BV's coefficient buffer column j; w <- w - V c.  onorm and norm
 * (host, nullable) receive ||w|| before the pass and sqrt(||w||^2 - c^T c),
 * or the explicit norm of the updated vector when that estimate is not
 * positive (bvorthog.c:124-127); asking for either synchronises the stream.
 * B200_ERR_INNER when w^T w < -10 eps for a column (BV_SafeSqrt). */
b200_status b200_bv_gram_schmidt(b200_bv bv, int j, double *v_dev, double *h_dev, double *c_dev, double *onorm,
                                 double *norm);
/* BVResize (src/sys/classes/bv/interface/bvbasic.c:338; BVResize_Svec,
 * impls/svec/svec.c:261): m columns of new storage, the first min(m, old m)
 * copied when copy != 0; l and k clipped to m.  The handle stays valid. */
b200_status b200_bv_resize(b200_bv bv, int m, int copy);
/* BVCopy (bvbasic.c:1779; BVCopy_Svec svec.c:233): Y(:, Y.l + j) =
 * X(:, X.l + j) for the k - l active columns of X. */
b200_status b200_bv_copy(b200_bv X, b200_bv Y);
/* BVNormalize (src/sys/classes/bv/interface/bvglobal.c:829) for real
 * scalars: every active column scaled to unit 2-norm (zero columns left as
 * they are); norms_host (nullable, k - l values) receives the norms. */
b200_status b200_bv_normalize(b200_bv bv, double *norms_host);
/* BVMultInPlaceHermitianTranspose (src/sys/classes/bv/interface/bvops.c:268)
 * for real scalars: V(:,s:e) = V(:,l:k) Q(s:e, l:k)^T with Q a host
 * column-major matrix of at least e rows (ldq >= e) and k columns. */
b200_status b200_bv_mult_inplace_trans(b200_bv bv, const double *Q_host, int ldq, int s, int e);
/* Allocation-free variant of b200_bv_orthogonalize_column; it has no
 * counterpart in SLEPc.  For callers that cannot call cudaMalloc -- for
 * example a host whose device memory is all owned by its own pool
 * allocator, or a plugin that must not grow the process's device footprint
 * after start-up.  V_dev is a caller-owned column-major basis (n rows,
 * leading dimension ld, even and >= n, ncols columns, 16-byte aligned);
 * column j is orthogonalised in place against columns 0..j-1 with the same
 * CGS + DGKS passes.  H_dev (device, j+1 doubles) receives the coefficients
 * and then the norm; norm and lindep (host, nullable) are read back, so the
 * call synchronises the stream.  All working memory comes from one fixed
 * array of about 330 KB compiled into the library, which every GPU that
 * loads the library holds until the process exits; j at most 253, otherwise
 * B200_ERR_ARG.  The first call on a device (and in each context of it the
 * caller makes current) looks the array's address up and should come before
 * any stream capture there.  The address is not looked up again after
 * cudaDeviceReset: do not call this entry point on a device after resetting
 * it.  Calls share the array: calls whose work overlaps on the GPU race and
 * must be serialised by the caller. */
b200_status b200_orthogonalize_column_noalloc(int n, int ld, int ncols, double *V_dev, int j, double *H_dev,
                                              double *norm, int *lindep, void *stream);
/* BVOrthogonalize (bvorthog.c:726-767) of columns l..k-1 with the BV's block
 * type: GS column by column (BVOrthogonalize_GS, :505-560); CHOL (:595-613) and
 * SVQB (:665-684) one Gram-Schmidt pass against columns 0..l-1, the Gram
 * matrix of the block on the device and its Cholesky factor or scaled
 * eigendecomposition on the host, then one in-place product.  R_host
 * (nullable, ldr >= k) receives R with V_in = V_out R (upper triangular
 * except for SVQB).  On B200_ERR_BREAKDOWN (a zero or linearly dependent
 * column) the status matches BVOrthogonalize_GS (bvorthog.c:546), but the
 * GS type queues every column before it reads any norm back, so the columns
 * after the dependent one have been processed too: the contents of columns
 * l..k-1 are undefined after a breakdown. */
b200_status b200_bv_orthogonalize(b200_bv bv, double *R_host, int ldr);

/* BVMultInPlace (bvops.c:220-245; BVMultInPlace_BLAS_CUDA bvcuda.cu:65-112):
 * V(:,s:e) = V(:,l:k) * Q(l:k,s:e) with the active columns l,k.  Q is a host
 * column-major matrix with leading dimension ldq (>= k). */
b200_status b200_bv_mult_inplace(b200_bv bv, const double *Q_host, int ldq, int s, int e);
/* Same with Q already in HBM. */
b200_status b200_bv_mult_inplace_device(b200_bv bv, const double *Q_dev, int ldq, int s, int e);
/* BVMult (bvops.c:47-85): Y(:,ly:ky) = alpha*X(:,lx:kx)*Q(lx:kx,ly:ky) + beta*Y(:,ly:ky). */
b200_status b200_bv_mult(b200_bv Y, double alpha, double beta, b200_bv X, const double *Q_host, int ldq);
/* BVMultVec (bvops.c:96-134): y = beta*y + alpha*X(:,l:k)*q, q_host of length k-l. */
b200_status b200_bv_mult_vec(b200_bv X, double alpha, double beta, double *y_dev, const double *q_host);
/* BVDot (bvglobal.c): M(ly:ky,lx:kx) = Y(:,ly:ky)^T X(:,lx:kx), M_host column-major ldm. */
b200_status b200_bv_dot(b200_bv X, b200_bv Y, double *M_host, int ldm);
/* BVDotVec (bvglobal.c): q = X(:,l:k)^T y, q_host of length k-l. */
b200_status b200_bv_dot_vec(b200_bv X, const double *y_dev, double *q_host);
/* BVScaleColumn / BVScale (bvops.c) -- j < 0 scales the active columns. */
b200_status b200_bv_scale_column(b200_bv bv, int j, double alpha);
/* BVNormColumn (NORM_2) and BVNorm (NORM_FROBENIUS of the active columns). */
b200_status b200_bv_norm_column(b200_bv bv, int j, double *nrm);
b200_status b200_bv_norm(b200_bv bv, double *nrm);
/* BVCopyColumn (bvops.c): column i <- column j. */
b200_status b200_bv_copy_column(b200_bv bv, int j, int i);
/* BVMatMult (bvops.c:692-730; matrix-product path of BVMatMult_Svec, svec.c:203-219):
 * Y(:, Y.l + j) = A V(:, V.l + j) for the active columns of V (Y has as many
 * active columns).  A square CSR operator is applied to all columns at once
 * (block SpMV: the matrix is read once, FP64 products and sums in index
 * order per row); other operators column by column. */
b200_status b200_bv_mat_mult(b200_bv V, b200_mat A, b200_bv Y);
/* BVMatMultColumn (bvops.c:862-890): column j+1 <- A * column j. */
b200_status b200_bv_mat_mult_column(b200_bv bv, b200_mat A, int j);
/* BVMatLanczos (src/sys/classes/bv/interface/bvkrylov.c:165-226): Lanczos
 * steps j = k..m-1 with full CGS+DGKS reorthogonalisation.  alpha_host and
 * beta_host (length >= m) receive T's diagonal and off-diagonal at k..m-1;
 * on breakdown m is reduced to the step that broke down. */
b200_status b200_bv_mat_lanczos(b200_bv bv, b200_mat A, int k, int *m, double *alpha_host, double *beta_host,
                                double *beta, int *breakdown);

/* ------------------------------------------------------------------ EPS --- */

/* EPSCreate + EPSSetType(EPSKRYLOVSCHUR) + EPSSetProblemType(EPS_HEP)
 * (src/eps/interface/epsbasic.c, src/eps/impls/krylov/krylovschur/krylovschur.c). */
b200_status b200_eps_create(void *stream, b200_eps *eps);
b200_status b200_eps_destroy(b200_eps eps);
/* EPSSetOperators(eps,A,NULL). */
b200_status b200_eps_set_operators(b200_eps eps, b200_mat A);
/* EPSSetDimensions (nev, ncv, mpd; ncv/mpd <= 0 take EPSSetDimensions_Default, epssetup.c:669-713). */
b200_status b200_eps_set_dimensions(b200_eps eps, int nev, int ncv, int mpd);
/* EPSSetTolerances (tol <= 0 -> 1e-8, slepcmath.h:25; max_it <= 0 -> max(100,2n/ncv), krylovschur.c:113). */
b200_status b200_eps_set_tolerances(b200_eps eps, double tol, int max_it);
/* EPSSetWhichEigenpairs (B200_LARGEST_MAGNITUDE ... B200_SMALLEST_REAL). */
b200_status b200_eps_set_which_eigenpairs(b200_eps eps, int which);
/* EPSKrylovSchurSetRestart (krylovschur.c:351-361), keep in [0.1,0.9]. */
b200_status b200_eps_krylovschur_set_restart(b200_eps eps, double keep);
/* EPSKrylovSchurSetLocking / GetLocking (krylovschur.c:427-500): lock = 1
 * (default) locks converged pairs at each restart; 0 selects the non-locking
 * variant (krylovschur.c:295: the kept vectors include the converged ones,
 * which stay in the active subspace), which needs mpd = ncv (krylovschur.c:116,
 * B200_ERR_SUP otherwise).  The mixed-precision form, a block method, ignores it. */
b200_status b200_eps_krylovschur_set_locking(b200_eps eps, int lock);
b200_status b200_eps_krylovschur_get_locking(b200_eps eps, int *lock);
/* EPSSetInitialSpace with one vector (epssetup.c:613, inserted at setup by BVInsertVecs). */
b200_status b200_eps_set_initial_space(b200_eps eps, const double *v0_host);
b200_status b200_eps_set_initial_space_device(b200_eps eps, const double *v0_dev);
/* Stop after this many restarts (0 = no cap; used to time bounded samples). */
b200_status b200_eps_set_max_restarts(b200_eps eps, int max_restarts);
/* EPSSolve (src/eps/interface/epssolve.c:119-229 -> EPSSolve_KrylovSchur_Default, krylovschur.c:227-348). */
/* Arithmetic of the Hermitian solve (no SLEPc counterpart: SLEPc computes in
 * the one precision PETSc was configured with).
 *   B200_PRECISION_FP64 (default): the drop-in path, Krylov-Schur in FP64
 *   throughout, as EPSSolve_KrylovSchur_Default.
 *   B200_PRECISION_MIXED: the same eigenpairs (every wanted residual
 *   ||Ax - theta x|| / |theta| below tol, computed in FP64 with the FP64
 *   matrix) by Chebyshev-filtered subspace iteration on a block of 64 or 128
 *   vectors (nev + guard), stored row-major, in two phases.  (1) FP32: the
 *   block and the matrix values in FP32, the filter's block SpMV accumulating
 *   in FP32, the orthonormalisation Gram matrix X^T X on the tensor cores
 *   (tcgen05 TF32 with FP32 accumulation) and the Rayleigh quotients X^T X,
 *   X^T A X and the residual norms in FP64, until tol_low.  (2) FP64: the same
 *   sweeps on the block widened to FP64 until tol.  The degree of each sweep
 *   follows the residuals and Ritz values.  Needs a square CSR operator,
 *   n >= 2 x block width, and which = largest/smallest real or largest
 *   magnitude. */
#define B200_PRECISION_FP64 0
#define B200_PRECISION_MIXED 1
b200_status b200_eps_set_precision(b200_eps eps, int precision);
/* The mixed form's projection kernel, exposed for tests and benchmarks (no
 * SLEPc counterpart as a call; it plays BVDot's role, bvglobal.c, on the
 * block): G (bp x bp, FP64, row-major, device) = X^T Y for row-major FP32
 * blocks of n rows and bp = 64 or 128 columns (Y null: X^T X).
 * tensor_cores = 1: tcgen05 kind::tf32 with FP32 accumulation in TMEM (the
 * TF32 inputs carry 10 mantissa bits); 0: FP64 products and sums on the CUDA
 * cores.  Allocates its work arrays; synchronises the stream. */
b200_status b200_rowblock_gram(int n, int bp, const float *X_dev, const float *Y_dev, int tensor_cores,
                               double *G_dev, void *stream);
/* The mixed form's filter step, exposed for tests and benchmarks: on row-major
 * device blocks of n rows and bp = 64 or 128 columns (FP32 when x32 = 1, with
 * the operator's values in FP32; FP64 otherwise), Y = alpha (A X - shift X)
 * - beta Z (Z nullable: no beta term) with the sliced-ELL block SpMV (products
 * accumulated in the block's precision, the affine update in FP64).  Builds
 * the operator's sliced-ELL and FP32 copies on first use; synchronises. */
b200_status b200_rowblock_spmm(b200_mat A, int bp, int x32, const void *X_dev, const void *Z_dev, void *Y_dev,
                               double alpha, double shift, double beta, void *stream);
/* The neural operator's contraction kernel, exposed for tests and benchmarks:
 * C[z] = alpha A[z] B[z] + beta C[z] for z < batch on device FP32 views
 * (A m x k, B k x n, C m x n; element (i, j) of matrix z of a view at
 * p + z*bs + i*rs + j*cs, any strides).  tcgen05 kind::tf32 MMAs, three per
 * step (high and low TF32 parts), FP32 accumulation in TMEM: FP32-level
 * accuracy.  split = 1 lets long depths split across CTAs (partial tiles
 * summed in a fixed order); sum_batch = 1 writes the single sum over z into
 * C (bsc ignored).  Allocates its work arrays; synchronises the stream. */
b200_status b200_tc_sgemm(int batch, int m, int n, int k, float alpha, const float *A_dev, long long ars,
                          long long acs, long long abs_, const float *B_dev, long long brs, long long bcs,
                          long long bbs, float beta, float *C_dev, long long rsc, long long csc, long long bsc,
                          int split, int sum_batch, void *stream);
/* The same product queued on the stream without allocation or synchronisation: the caller passes
 * the split-depth workspace (ws_floats floats, null for none: no depth split, and sum_batch then
 * not allowed) and a device int that collects the error bits of bounded waits (read it after a
 * synchronisation; nonzero means the product is invalid). */
b200_status b200_tc_sgemm_async(int batch, int m, int n, int k, float alpha, const float *A_dev, long long ars,
                                long long acs, long long abs_, const float *B_dev, long long brs, long long bcs,
                                long long bbs, float beta, float *C_dev, long long rsc, long long csc, long long bsc,
                                int sum_batch, float *ws_dev, size_t ws_floats, int *err_dev, void *stream);
/* Mixed-form parameters (0 or a negative value keeps the default): tol_low,
 * the tolerance of the FP32 phase (default 5e-7, never below tol; the phase
 * also ends when a sweep no longer halves the largest wanted residual);
 * degree, the largest Chebyshev degree of one sweep (default 400; a sweep
 * runs in segments, each followed by an orthonormalisation); guard,
 * block columns beyond nev (default max(8, nev/2); the block is 64 columns
 * when nev + guard <= 64, else 128, at most 128); max_sweeps, per phase
 * (default 60); fp64_gram: 1 forms the FP32 phase's orthonormalisation Gram
 * matrix in FP64 (FP64 MMAs) instead of in TF32 on the tcgen05 tensor cores
 * (0, default). */
b200_status b200_eps_set_mixed_options(b200_eps eps, double tol_low, int degree, int guard, int max_sweeps,
                                       int fp64_gram);

/* EPSSetType: B200_EPS_KRYLOVSCHUR (default) or B200_EPS_LOBPCG. */
#define B200_EPS_KRYLOVSCHUR 0
#define B200_EPS_LOBPCG 1
b200_status b200_eps_set_type(b200_eps eps, int type);
/* EPSLOBPCGSetBlockSize (bs <= 0: min(16, nev)), EPSLOBPCGSetRestart (in [0.1, 1]),
 * EPSLOBPCGSetLocking (src/eps/impls/cg/lobpcg/lobpcg.c). */
b200_status b200_eps_lobpcg_set_block_size(b200_eps eps, int bs);
b200_status b200_eps_lobpcg_set_restart(b200_eps eps, double restart);
b200_status b200_eps_lobpcg_set_locking(b200_eps eps, int lock);
/* Preconditioner of a preconditioned eigensolver: STPRECOND with KSPPREONLY and
 * PCNONE (identity) or PCJACOBI (diag(A)^{-1}, a zero diagonal entry counts as 1). */
#define B200_PC_NONE 0
#define B200_PC_JACOBI 1
b200_status b200_eps_set_preconditioner(b200_eps eps, int pc);
/* BVSetOrthogonalization block type of the eigensolver's basis (-bv_orthog_block),
 * which LOBPCG's X, R and P blocks inherit (lobpcg.c:256, :331, :334 call
 * BVOrthogonalize on them).  Krylov-Schur orthogonalises column by column and
 * does not use it. */
b200_status b200_eps_set_bv_orthog_block(b200_eps eps, int type);
/* EPSSetInitialSpace with k vectors (host, n x k column-major): inserted and
 * orthonormalised as BVInsertVecs does, linearly dependent ones dropped
 * (src/sys/classes/bv/interface/bvfunc.c:331-374).  Krylov-Schur starts from
 * the first; LOBPCG uses the block. */
b200_status b200_eps_set_initial_space_block(b200_eps eps, int k, const double *X_host);
b200_status b200_eps_solve(b200_eps eps);
b200_status b200_eps_get_converged(b200_eps eps, int *nconv);
b200_status b200_eps_get_iteration_number(b200_eps eps, int *its);
b200_status b200_eps_get_converged_reason(b200_eps eps, int *reason);
/* EPSGetEigenpair (epssolve.c:406): eigenvalue and (nullable) eigenvector copied to the host. */
b200_status b200_eps_get_eigenpair(b200_eps eps, int i, double *eigr, double *x_host);
/* Device address of the i-th eigenvector (valid until the next solve). */
b200_status b200_eps_get_eigenvector_device(b200_eps eps, int i, const double **x_dev);
/* EPSGetErrorEstimate (epssolve.c) and EPSComputeError (epssolve.c:742-838). */
b200_status b200_eps_get_error_estimate(b200_eps eps, int i, double *errest);
b200_status b200_eps_compute_error(b200_eps eps, int i, int type, double *error);
/* Counters of the last solve: Lanczos steps, Gram-Schmidt passes that did
 * work, restarts, kernels launched, algorithmic bytes of the Gram-Schmidt
 * passes, and device time of each kernel family (ms, CUDA events; the
 * per-family times are 0 unless timing is on). */
typedef struct {
  int64_t lanczos_steps;
  int64_t gs_passes;
  int64_t restarts;
  int64_t kernel_launches;
  double ms_spmv, ms_orth, ms_restart, ms_total;
  int64_t gs_bytes;
  int64_t column_visits;  /* sum over Lanczos steps j of (j+2): basis columns one CGS pass reads */
  /* mixed precision (zero otherwise): sweeps of the FP64 phase, the largest Chebyshev degree of a
   * sweep, block columns, sweeps of the FP32 phase, device time of the two phases, and block-SpMV
   * columns (block width x block SpMVs).  In the mixed form gs_passes counts the block
   * orthonormalisations (SVQB) and restarts the Rayleigh-Ritz steps; with timing on, ms_spmv and
   * gs_bytes hold the device time and the algorithmic bytes of the Chebyshev filters' block SpMVs,
   * ms_orth and ms_restart the wall time of the orthonormalisations and Rayleigh-Ritz steps. */
  int64_t filter_sweeps;
  int64_t filter_degree;
  int64_t block_size;
  int64_t phase1_restarts;
  double ms_phase1, ms_phase2;
  int64_t spmm_columns;
} b200_eps_stats;
b200_status b200_eps_get_stats(b200_eps eps, b200_eps_stats *stats);
/* Enable per-phase CUDA-event timing (adds events around each phase). */
b200_status b200_eps_set_timing(b200_eps eps, int on);

/* EPSMonitorSet (src/eps/interface/epsmon.c:96) / EPSMonitorCancel: a monitor
 * is called on the host once per outer iteration, where EPSSolve_KrylovSchur
 * calls EPSMonitor (krylovschur.c:339; for the mixed form, once per sweep),
 * with the iteration number, the number of converged pairs, the current Ritz
 * values and error estimates and their count (real scalars: no eigi).  Up to
 * 8 monitors; a nonzero return aborts the solve with B200_ERR_STATE.
 * b200_eps_monitor_jsonl adds a built-in monitor writing one JSON line per
 * iteration to path: its, nconv, nest, eigr, errest, the host milliseconds
 * since the solve started and the Gram-Schmidt algorithmic bytes so far. */
typedef int (*b200_eps_monitor_fn)(b200_eps eps, int its, int nconv, const double *eigr, const double *errest,
                                   int nest, void *ctx);
b200_status b200_eps_monitor_set(b200_eps eps, b200_eps_monitor_fn fn, void *ctx);
b200_status b200_eps_monitor_cancel(b200_eps eps);
b200_status b200_eps_monitor_jsonl(b200_eps eps, const char *path);

/* One call from host buffers to host results: create the matrix, solve,
 * copy eigenvalues (nconv), eigenvectors (n x nconv column-major, nullable)
 * and error estimates (nullable) back.  info_host[0..4] = nconv, its,
 * reason, lanczos steps, restarts.  This is the end-to-end entry point that
 * an EPSSolve caller with host data would bind. */
b200_status b200_eps_solve_csr_host(int n, int64_t nnz, const int *rowptr_host, const int *colind_host,
                                    const double *vals_host, const double *v0_host, int nev, int ncv, int mpd,
                                    double tol, int max_it, int which, double *evals_host, double *X_host,
                                    double *errest_host, int *info_host, void *stream);
/* The same with the arithmetic form chosen (B200_PRECISION_FP64 or
 * B200_PRECISION_MIXED, b200_eps_set_precision); X_host then needs room for
 * nconv vectors, at most max(ncv, 128). */
b200_status b200_eps_solve_csr_host_ex(int n, int64_t nnz, const int *rowptr_host, const int *colind_host,
                                       const double *vals_host, const double *v0_host, int nev, int ncv, int mpd,
                                       double tol, int max_it, int which, int precision, double *evals_host,
                                       double *X_host, double *errest_host, int *info_host, void *stream);

/* ----------------------------------------------------- PETSc binary I/O --- */

/* The PETSc binary format of MatView/VecView and MatLoad/VecLoad
 * (PetscViewerBinaryOpen as used by src/eps/tutorials/ex4.c:45-48 and
 * ex31.c:551-562): big-endian, 32-bit PetscInt, real double PetscScalar.
 *   Mat: int32 classid 1211216, M, N, nz, row lengths[M], column indices[nz], float64 values[nz]
 *   Vec: int32 classid 1211214, N, float64 values[N]
 * Objects follow one another in a file.  PetscViewerBinaryOpen / PetscViewerDestroy: */
b200_status b200_viewer_binary_open(const char *path, int mode, b200_viewer *v);
b200_status b200_viewer_destroy(b200_viewer v);
/* Header of the next object without consuming it: classid, and M, N, nz for a
 * Mat or N, 1, N for a Vec.  B200_ERR_IO at the end of the file. */
b200_status b200_viewer_peek(b200_viewer v, int *classid, int *m, int *n, int64_t *nnz);
/* Read the next Mat into host CSR arrays (rowptr M+1, colind/vals nz, sizes from peek). */
b200_status b200_mat_read_csr(b200_viewer v, int *rowptr_host, int *colind_host, double *vals_host);
b200_status b200_mat_write_csr(b200_viewer v, int m, int n, int64_t nnz, const int *rowptr_host,
                               const int *colind_host, const double *vals_host);
/* VecLoad / VecView of host arrays (nmax: capacity of x_host; n: length read). */
b200_status b200_vec_read(b200_viewer v, int nmax, int *n, double *x_host);
b200_status b200_vec_write(b200_viewer v, int n, const double *x_host);
/* MatLoad into HBM (storage B200_MAT_OPERATOR, B200_SCALAR_F64 or B200_SCALAR_F32) and MatView. */
b200_status b200_mat_load(b200_viewer v, int storage, void *stream, b200_mat *A);
b200_status b200_mat_view(b200_mat A, b200_viewer v);

/* ------------------------------------------------------------------ SVD --- */

/* The SVD cross solver (SVDCROSS, src/svd/impls/cross/cross.c) for a standard
 * problem: Krylov-Schur (the b200_eps solver above) on the shell A^T A of
 * b200_mat_create_cross, sigma = sqrt(lambda), left vectors U = A V
 * orthogonalised by Gram-Schmidt.  A comes from b200_mat_create_aij; when A
 * has fewer rows than columns the operator is A A^T and the roles of U and V
 * are exchanged, as SVDSetUp does (src/svd/interface/svdsetup.c:300-343).
 * SVDCreate / SVDDestroy / SVDSetOperators(svd,A,NULL). */
b200_status b200_svd_create(void *stream, b200_svd *svd);
b200_status b200_svd_destroy(b200_svd svd);
b200_status b200_svd_set_operator(b200_svd svd, b200_mat A);
/* SVDSetDimensions (ncv, mpd <= 0: the EPS defaults). */
b200_status b200_svd_set_dimensions(b200_svd svd, int nsv, int ncv, int mpd);
/* SVDSetTolerances (tol <= 0: 1e-8, and the EPS runs with 1e-9 as
 * SVDSetUp_Cross chooses, cross.c:217; max_it <= 0: the EPS default). */
b200_status b200_svd_set_tolerances(b200_svd svd, double tol, int max_it);
/* SVDSetWhichSingularTriplets: B200_SVD_LARGEST or B200_SVD_SMALLEST. */
b200_status b200_svd_set_which_singular_triplets(b200_svd svd, int which);
/* SVDSetInitialSpaces with one vector, of the operator's dimension: the
 * columns of A, or its rows when A has fewer rows than columns (the spaces
 * are swapped with the matrix, svdsetup.c:333-338). */
b200_status b200_svd_set_initial_space(b200_svd svd, const double *v0_host);
/* Per-phase CUDA-event timing of the inner eigensolve (b200_eps_set_timing). */
b200_status b200_svd_set_timing(b200_svd svd, int on);
/* SVDSolve (src/svd/interface/svdsolve.c) with SVDSolve_Cross (cross.c:256-285). */
b200_status b200_svd_solve(b200_svd svd);
b200_status b200_svd_get_converged(b200_svd svd, int *nconv);
b200_status b200_svd_get_iteration_number(b200_svd svd, int *its);
b200_status b200_svd_get_converged_reason(b200_svd svd, int *reason);
/* SVDGetSingularTriplet: sigma_i and (nullable) host copies of u_i (length m)
 * and v_i (length n).  The singular vectors are computed on first request
 * (SVDComputeVectors_Cross, cross.c:287-355). */
b200_status b200_svd_get_singular_triplet(b200_svd svd, int i, double *sigma, double *u_host, double *v_host);
/* Device addresses of u_i and v_i, valid until the next solve or destroy. */
b200_status b200_svd_get_singular_vectors_device(b200_svd svd, int i, const double **u_dev, const double **v_dev);
/* SVDComputeError (svdsolve.c:485-580): sqrt(||A v - sigma u||^2 + ||A^T u - sigma v||^2),
 * divided by sigma*sqrt(2) (B200_ERROR_RELATIVE) or ||A||_inf*sqrt(2) (B200_ERROR_NORM). */
b200_status b200_svd_compute_error(b200_svd svd, int i, int type, double *error);
/* Statistics of the inner Krylov-Schur solve. */
b200_status b200_svd_get_stats(b200_svd svd, b200_eps_stats *stats);

/* One call from host CSR to host singular triplets, largest first:
 * sigma_host (nconv values), U_host (m x nconv, column-major), V_host
 * (n x nconv), rel_error_host (relative errors), all nullable; info_host[0..4]
 * = nconv, its, reason, lanczos steps, restarts. */
b200_status b200_svd_solve_aij_host(int m, int n, int64_t nnz, const int *rowptr_host, const int *colind_host,
                                    const void *vals_host, int scalar_type, const double *v0_host, int nsv, int ncv,
                                    double tol, int max_it, double *sigma_host, double *U_host, double *V_host,
                                    double *rel_error_host, int *info_host, void *stream);

/* ---------------------------------------------------- learned warm start --- */

/* A spectral neural operator that maps the coefficient field of a diffusion
 * operator on an N x N grid to nout fields, trained to reproduce the
 * operator's lowest eigenvectors; its output is a starting block for
 * EPSSetInitialSpace (src/eps/interface/epssetup.c:613), the hook through
 * which a SLEPc user supplies an initial space (no network exists in SLEPc).
 * Forward, backward and the Adam update run in this library's own FP32
 * kernels.  Inputs per sample: 3 x N*N features (log kappa, x, y of the cell
 * centres, row-major); outputs nout x N*N.  Network: pointwise lift to
 * `width` channels, `layers` layers of (Dirichlet sine-mode spectral mixing
 * over modes x modes modes + pointwise mixing, gelu), pointwise projection
 * through `hidden` channels.  Loss per output k: 1 - (y_k . u_k)^2 / |y_k|^2
 * against a unit target u_k, averaged.  Parameters are one flat FP32 array
 * (set/get from host memory; initialisation is the caller's). */
typedef struct b200_neural_op_s *b200_neural_op;
b200_status b200_neural_op_create(int N, int width, int modes, int layers, int hidden, int nout, void *stream,
                                  b200_neural_op *op);
b200_status b200_neural_op_destroy(b200_neural_op op);
b200_status b200_neural_op_num_params(b200_neural_op op, int64_t *n);
b200_status b200_neural_op_set_params(b200_neural_op op, const float *params_host);  /* also resets Adam */
b200_status b200_neural_op_get_params(b200_neural_op op, float *params_host);
/* out_dev (batch x nout x N*N) = network(features_dev (batch x 3 x N*N)), device pointers */
b200_status b200_neural_op_forward(b200_neural_op op, int batch, const float *features_dev, float *out_dev);
/* mean loss against targets_dev (batch x nout x N*N) */
b200_status b200_neural_op_loss(b200_neural_op op, int batch, const float *features_dev, const float *targets_dev,
                                float *loss);
/* loss and its gradient with respect to every parameter (grads_host nullable, nparams floats) */
b200_status b200_neural_op_loss_grad(b200_neural_op op, int batch, const float *features_dev,
                                     const float *targets_dev, float *loss, float *grads_host);
/* one Adam step (beta1 0.9, beta2 0.999, eps 1e-8) on the loss of one batch */
b200_status b200_neural_op_train_step(b200_neural_op op, int batch, const float *features_dev,
                                      const float *targets_dev, float lr, float *loss);

/* -------------------------------------------------------------- batched --- */

/* Many independent small Hermitian eigenproblems solved by Krylov-Schur in one
 * persistent launch (no SLEPc counterpart as one call: it stands for a loop
 * of EPSSolve over the problems).  Each CTA of the launch takes a problem
 * from a work queue (largest first) and runs the whole solve for it on the
 * device: Lanczos with CGS+DGKS, the projected problem (implicit QL in place
 * of LAPACK dsteqr), sort, convergence test, truncation and the restart.
 * The launch is captured in a CUDA graph and replayed; the CTA size is
 * chosen by an autotuner unless set.
 *   rowptr: the problems' row pointers one after another (ns[p]+1 local
 *   offsets each); colind (local indices) and vals: their nonzeros one after
 *   another; rows of at most 256 nonzeros.  Copied to HBM. */
b200_status b200_batch_create(int nprob, const int *ns_host, const int *rowptr_host, const int *colind_host,
                              const double *vals_host, void *stream, b200_batch *B);
b200_status b200_batch_destroy(b200_batch B);
/* EPSSetDimensions for every problem (ncv <= 31; ncv <= the smallest n). */
b200_status b200_batch_set_dimensions(b200_batch B, int nev, int ncv, int mpd);
b200_status b200_batch_set_tolerances(b200_batch B, double tol, int max_it);
b200_status b200_batch_set_which_eigenpairs(b200_batch B, int which);
/* Start vectors, one after another (sum of ns doubles); all zero by default,
 * which means random starts (a zero initial vector is dropped). */
b200_status b200_batch_set_initial_vectors(b200_batch B, const double *v0_host);
/* CTA size per problem: 128, 256, 512, or 0 for the autotuner (default). */
b200_status b200_batch_set_threads(b200_batch B, int threads);
/* Times each CTA size on the largest problems and keeps the fastest. */
b200_status b200_batch_autotune(b200_batch B, int *threads);
b200_status b200_batch_solve(b200_batch B);
/* Results of problem p: converged count, restarts, reason, Lanczos steps, and the
 * sorted eigenvalues / error estimates (nconv values each, nullable). */
b200_status b200_batch_get_solution(b200_batch B, int p, int *nconv, int *its, int *reason, int *lanczos_steps,
                                    double *evals_host, double *errest_host);
b200_status b200_batch_get_eigenvector(b200_batch B, int p, int i, double *x_host);
/* All results at once: evals_host (nprob x ncv), info_host (nprob x 8: nconv, its, reason,
 * steps, device error), and the device time of the last solve in ms. */
b200_status b200_batch_get_all(b200_batch B, double *evals_host, int *info_host, float *ms);
/* Algorithmic bytes the last solve moved (SpMV: 12 per nonzero plus the vectors; Gram-Schmidt
 * dots and updates: 8 per row and column touched; restarts), summed over the problems. */
b200_status b200_batch_get_bytes(b200_batch B, double *bytes);
/* Precision of the batched solve (no SLEPc counterpart).  B200_PRECISION_FP64 (default);
 * B200_PRECISION_MIXED: phase 1 runs the same per-problem Krylov-Schur with every basis stored in
 * FP32 (FP64 work vector, products and sums; half the basis bytes) to tol_low (default 1e-6);
 * phase 2 runs the FP64 solve of each problem from the sum of its phase-1 Ritz vectors to tol.
 * The three launches (phase 1, start vectors, phase 2) form one captured graph; the results are
 * phase 2's.  get_bytes then counts both phases. */
b200_status b200_batch_set_precision(b200_batch B, int precision, double tol_low);
/* Phase-1 counters of the last mixed solve: info_host (nprob x 8, as get_all) and its bytes. */
b200_status b200_batch_get_phase1(b200_batch B, int *info_host, double *bytes);

#ifdef __cplusplus
}
#endif

#endif /* SLEPC_B200_H */
