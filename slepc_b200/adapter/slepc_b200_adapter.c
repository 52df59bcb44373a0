/*
 * SLEPc adapter for the B200 Krylov-Schur library.
 *
 * Compiled inside a SLEPc build (PETSc configured with CUDA, real double
 * scalars, 32-bit PetscInt); it is not compiled in this repository's image,
 * which has no PETSc.  It registers:
 *
 *   BV type  "b200"    BVRegister("b200", BVCreate_B200)     (bv/interface/bvfunc.c:646)
 *   EPS type "b200ks"  EPSRegister("b200ks", EPSCreate_B200KS) (eps/interface/epsbasic.c:235)
 *
 * and provides MatCreateB200(aij, &shell), a MATSHELL whose MatMult is the
 * B200 CSR SpMV on VECCUDA arrays (precedent: MatMult_Cyclic_CUDA in
 * src/svd/impls/cyclic/cycliccuda/cycliccuda.cu:16-48).
 *
 * The BV type keeps SLEPc's own DGKS driver (BVOrthogonalizeGS, bvorthog.c:145-217)
 * and fills its gramschmidt op (bvimpl.h:53) with b200_bv_gram_schmidt, so a
 * stock EPSSolve with -bv_type b200 alone runs every Gram-Schmidt pass on the
 * device pass kernel.  The optional EPS type hands a whole Hermitian solve to
 * b200_eps_solve, which also fuses the DGKS passes and keeps a Lanczos run on
 * the device with one host synchronisation.
 */
#include <slepc/private/bvimpl.h>
#include <slepc/private/epsimpl.h>
#include <petscdevice_cuda.h>

#include "slepc_b200.h"

static PetscErrorCode B200ToPetsc(b200_status s)
{
  switch (s) {
  case B200_OK:            return PETSC_SUCCESS;
  case B200_ERR_ARG:       return PETSC_ERR_ARG_OUTOFRANGE;
  case B200_ERR_CUDA:      return PETSC_ERR_GPU;
  case B200_ERR_LAPACK:    return PETSC_ERR_LIB;
  case B200_ERR_INNER:     return PETSC_ERR_USER_INPUT;
  case B200_ERR_BREAKDOWN: return PETSC_ERR_CONV_FAILED;
  case B200_ERR_NOMEM:     return PETSC_ERR_MEM;
  case B200_ERR_STATE:     return PETSC_ERR_ORDER;
  default:                 return PETSC_ERR_LIB;
  }
}

#define B200Call(expr) \
  do { \
    b200_status _s = (expr); \
    PetscCheck(_s == B200_OK, PETSC_COMM_SELF, B200ToPetsc(_s), "slepc_b200: %s", b200_last_error()); \
  } while (0)

/* ------------------------------------------------------------------ Mat --- */

typedef struct {
  b200_mat A;
} Mat_B200;

static PetscErrorCode MatMult_B200(Mat S, Vec x, Vec y)
{
  Mat_B200          *ctx;
  const PetscScalar *px;
  PetscScalar       *py;

  PetscFunctionBegin;
  PetscCall(MatShellGetContext(S, &ctx));
  PetscCall(VecCUDAGetArrayRead(x, &px));
  PetscCall(VecCUDAGetArrayWrite(y, &py));
  B200Call(b200_mat_mult(ctx->A, px, py));
  PetscCall(VecCUDARestoreArrayRead(x, &px));
  PetscCall(VecCUDARestoreArrayWrite(y, &py));
  PetscFunctionReturn(PETSC_SUCCESS);
}

static PetscErrorCode MatDestroyContext_B200(void *c)
{
  Mat_B200 *ctx = (Mat_B200 *)c;

  PetscFunctionBegin;
  B200Call(b200_mat_destroy(ctx->A));
  PetscCall(PetscFree(ctx));
  PetscFunctionReturn(PETSC_SUCCESS);
}

/* Wrap an assembled MATSEQAIJ: its CSR arrays are copied to HBM once. */
PetscErrorCode MatCreateB200(Mat aij, Mat *S)
{
  Mat_B200          *ctx;
  PetscInt           n, nr;
  const PetscInt    *ia, *ja;
  const PetscScalar *va;
  PetscBool          done;

  PetscFunctionBegin;
  PetscCheck(sizeof(PetscInt) == sizeof(int), PETSC_COMM_SELF, PETSC_ERR_SUP, "needs 32-bit PetscInt");
  PetscCall(MatGetSize(aij, &n, NULL));
  PetscCall(PetscNew(&ctx));
  PetscCall(MatGetRowIJ(aij, 0, PETSC_FALSE, PETSC_FALSE, &nr, &ia, &ja, &done));
  PetscCheck(done, PETSC_COMM_SELF, PETSC_ERR_SUP, "MatGetRowIJ failed");
  PetscCall(MatSeqAIJGetArrayRead(aij, &va));
  B200Call(b200_mat_create_csr((int)n, (int64_t)ia[n], (const int *)ia, (const int *)ja, va, NULL, &ctx->A));
  PetscCall(MatSeqAIJRestoreArrayRead(aij, &va));
  PetscCall(MatRestoreRowIJ(aij, 0, PETSC_FALSE, PETSC_FALSE, &nr, &ia, &ja, &done));
  PetscCall(MatCreateShell(PETSC_COMM_SELF, n, n, n, n, ctx, S));
  PetscCall(MatShellSetOperation(*S, MATOP_MULT, (void (*)(void))MatMult_B200));
  PetscCall(MatShellSetOperation(*S, MATOP_MULT_TRANSPOSE, (void (*)(void))MatMult_B200)); /* symmetric */
  PetscCall(MatShellSetContextDestroy(*S, MatDestroyContext_B200));
  PetscCall(MatShellSetVecType(*S, VECCUDA));
  PetscCall(PetscObjectChangeTypeName((PetscObject)*S, "b200csr"));
  PetscFunctionReturn(PETSC_SUCCESS);
}

static PetscErrorCode MatB200Get(Mat S, b200_mat *A)
{
  PetscBool  is;
  Mat_B200  *ctx;

  PetscFunctionBegin;
  PetscCall(PetscObjectTypeCompare((PetscObject)S, "b200csr", &is));
  *A = NULL;
  if (is) {
    PetscCall(MatShellGetContext(S, &ctx));
    *A = ctx->A;
  }
  PetscFunctionReturn(PETSC_SUCCESS);
}

/* ------------------------------------------------------------------- BV --- */

typedef struct {
  b200_bv bv;    /* device storage: ld x (m+1) doubles */
  Vec     v;     /* VECSEQCUDA over the storage (for getarray / getmat paths) */
  double *stage; /* device staging of the host h / c arrays of BVOrthogonalizeVec (2 (m+1) doubles) */
  Mat     Aget;  /* dense CUDA matrix over the active columns (getmat / restoremat) */
} BV_B200;

/* the ABI keeps its own active columns; mirror SLEPc's before every op */
static PetscErrorCode BVB200Sync(BV bv)
{
  BV_B200 *ctx = (BV_B200 *)bv->data;

  PetscFunctionBegin;
  PetscCheck(!bv->nc, PetscObjectComm((PetscObject)bv), PETSC_ERR_SUP, "BV b200: constraints not supported");
  B200Call(b200_bv_set_active_columns(ctx->bv, bv->l, bv->k));
  PetscFunctionReturn(PETSC_SUCCESS);
}

static PetscErrorCode BVMultInPlace_B200(BV V, Mat Q, PetscInt s, PetscInt e)
{
  BV_B200           *ctx = (BV_B200 *)V->data;
  const PetscScalar *q;
  PetscInt           ldq;

  PetscFunctionBegin;
  PetscCall(BVB200Sync(V));
  PetscCall(MatDenseGetLDA(Q, &ldq));
  PetscCall(MatDenseGetArrayRead(Q, &q));
  B200Call(b200_bv_mult_inplace(ctx->bv, q, (int)ldq, (int)s, (int)e));
  PetscCall(MatDenseRestoreArrayRead(Q, &q));
  PetscFunctionReturn(PETSC_SUCCESS);
}

static PetscErrorCode BVMult_B200(BV Y, PetscScalar alpha, PetscScalar beta, BV X, Mat Q)
{
  BV_B200           *y = (BV_B200 *)Y->data, *x = (BV_B200 *)X->data;
  const PetscScalar *q;
  PetscInt           ldq;

  PetscFunctionBegin;
  PetscCheck(Q, PetscObjectComm((PetscObject)Y), PETSC_ERR_SUP, "BV b200: BVMult without Q not supported");
  PetscCall(BVB200Sync(Y));
  PetscCall(BVB200Sync(X));
  PetscCall(MatDenseGetLDA(Q, &ldq));
  PetscCall(MatDenseGetArrayRead(Q, &q));
  B200Call(b200_bv_mult(y->bv, alpha, beta, x->bv, q, (int)ldq));
  PetscCall(MatDenseRestoreArrayRead(Q, &q));
  PetscFunctionReturn(PETSC_SUCCESS);
}

/* q == NULL: coefficients live in bv->buffer (BVGetBufferVec, bvbasic.c:775-790) */
static PetscErrorCode BVMultVec_B200(BV X, PetscScalar alpha, PetscScalar beta, Vec y, PetscScalar *q)
{
  BV_B200     *ctx = (BV_B200 *)X->data;
  PetscScalar *py, *qq = q;

  PetscFunctionBegin;
  PetscCall(BVB200Sync(X));
  if (!q) PetscCall(VecGetArray(X->buffer, &qq));
  PetscCall(VecCUDAGetArray(y, &py));
  B200Call(b200_bv_mult_vec(ctx->bv, alpha, beta, py, qq));
  PetscCall(VecCUDARestoreArray(y, &py));
  if (!q) PetscCall(VecRestoreArray(X->buffer, &qq));
  PetscFunctionReturn(PETSC_SUCCESS);
}

static PetscErrorCode BVDotVec_B200(BV X, Vec y, PetscScalar *q)
{
  BV_B200           *ctx = (BV_B200 *)X->data;
  const PetscScalar *py;
  PetscScalar       *qq = q;

  PetscFunctionBegin;
  PetscCheck(!X->matrix, PetscObjectComm((PetscObject)X), PETSC_ERR_SUP, "BV b200: non-standard inner product");
  PetscCall(BVB200Sync(X));
  if (!q) PetscCall(VecGetArray(X->buffer, &qq));
  PetscCall(VecCUDAGetArrayRead(y, &py));
  B200Call(b200_bv_dot_vec(ctx->bv, py, qq));
  PetscCall(VecCUDARestoreArrayRead(y, &py));
  if (!q) PetscCall(VecRestoreArray(X->buffer, &qq));
  PetscFunctionReturn(PETSC_SUCCESS);
}

static PetscErrorCode BVDot_B200(BV X, BV Y, Mat M)
{
  BV_B200     *x = (BV_B200 *)X->data;
  BV_B200     *y = (BV_B200 *)Y->data;
  PetscScalar *m;
  PetscInt     ldm;

  PetscFunctionBegin;
  PetscCall(BVB200Sync(X));
  PetscCall(BVB200Sync(Y));
  PetscCall(MatDenseGetLDA(M, &ldm));
  PetscCall(MatDenseGetArray(M, &m));
  B200Call(b200_bv_dot(x->bv, y->bv, m, (int)ldm));
  PetscCall(MatDenseRestoreArray(M, &m));
  PetscFunctionReturn(PETSC_SUCCESS);
}

static PetscErrorCode BVScale_B200(BV bv, PetscInt j, PetscScalar alpha)
{
  BV_B200 *ctx = (BV_B200 *)bv->data;

  PetscFunctionBegin;
  PetscCall(BVB200Sync(bv));
  B200Call(b200_bv_scale_column(ctx->bv, (int)j, alpha));
  PetscFunctionReturn(PETSC_SUCCESS);
}

static PetscErrorCode BVNorm_B200(BV bv, PetscInt j, NormType type, PetscReal *val)
{
  BV_B200 *ctx = (BV_B200 *)bv->data;
  double   v;

  PetscFunctionBegin;
  PetscCall(BVB200Sync(bv));
  if (j >= 0) {
    PetscCheck(type == NORM_2, PetscObjectComm((PetscObject)bv), PETSC_ERR_SUP, "BV b200: column norms are 2-norms");
    B200Call(b200_bv_norm_column(ctx->bv, (int)j, &v));
  } else {
    PetscCheck(type == NORM_FROBENIUS, PetscObjectComm((PetscObject)bv), PETSC_ERR_SUP, "BV b200: Frobenius norm only");
    B200Call(b200_bv_norm(ctx->bv, &v));
  }
  *val = v;
  PetscFunctionReturn(PETSC_SUCCESS);
}

static PetscErrorCode BVCopyColumn_B200(BV bv, PetscInt j, PetscInt i)
{
  BV_B200 *ctx = (BV_B200 *)bv->data;

  PetscFunctionBegin;
  B200Call(b200_bv_copy_column(ctx->bv, (int)j, (int)i));
  PetscFunctionReturn(PETSC_SUCCESS);
}

static PetscErrorCode BVGetColumn_B200(BV bv, PetscInt j, Vec *v)
{
  BV_B200 *ctx = (BV_B200 *)bv->data;
  double  *V;
  PetscInt l = BVAvailableVec;

  PetscFunctionBegin;
  B200Call(b200_bv_get_array(ctx->bv, &V));
  PetscCall(VecCUDAPlaceArray(bv->cv[l], V + (bv->nc + j) * bv->ld));
  PetscFunctionReturn(PETSC_SUCCESS);
}

static PetscErrorCode BVRestoreColumn_B200(BV bv, PetscInt j, Vec *v)
{
  PetscInt l = (j == bv->ci[0]) ? 0 : 1;

  PetscFunctionBegin;
  PetscCall(VecCUDAResetArray(bv->cv[l]));
  PetscFunctionReturn(PETSC_SUCCESS);
}

static PetscErrorCode BVGetArray_B200(BV bv, PetscScalar **a)
{
  BV_B200 *ctx = (BV_B200 *)bv->data;

  PetscFunctionBegin;
  PetscCall(VecGetArray(ctx->v, a));
  PetscFunctionReturn(PETSC_SUCCESS);
}

static PetscErrorCode BVRestoreArray_B200(BV bv, PetscScalar **a)
{
  BV_B200 *ctx = (BV_B200 *)bv->data;

  PetscFunctionBegin;
  PetscCall(VecRestoreArray(ctx->v, a));
  PetscFunctionReturn(PETSC_SUCCESS);
}

static PetscErrorCode BVGetArrayRead_B200(BV bv, const PetscScalar **a)
{
  BV_B200 *ctx = (BV_B200 *)bv->data;

  PetscFunctionBegin;
  PetscCall(VecGetArrayRead(ctx->v, a));
  PetscFunctionReturn(PETSC_SUCCESS);
}

static PetscErrorCode BVRestoreArrayRead_B200(BV bv, const PetscScalar **a)
{
  BV_B200 *ctx = (BV_B200 *)bv->data;

  PetscFunctionBegin;
  PetscCall(VecRestoreArrayRead(ctx->v, a));
  PetscFunctionReturn(PETSC_SUCCESS);
}

static PetscErrorCode BVMatMult_B200(BV V, Mat A, BV W)
{
  PetscInt j;
  Vec      v, w;

  PetscFunctionBegin;
  for (j = 0; j < V->k - V->l; j++) {
    PetscCall(BVGetColumn(V, V->l + j, &v));
    PetscCall(BVGetColumn(W, W->l + j, &w));
    PetscCall(MatMult(A, v, w));
    PetscCall(BVRestoreColumn(W, W->l + j, &w));
    PetscCall(BVRestoreColumn(V, V->l + j, &v));
  }
  PetscFunctionReturn(PETSC_SUCCESS);
}

/* The gramschmidt op (bvimpl.h:53): one CGS pass through b200_bv_gram_schmidt, called 1-3 times
   by BVOrthogonalizeGS's DGKS loop (bvorthog.c:174-203) in place of BVOrthogonalizeCGS1.  Column
   variant (v NULL): SLEPc passes h = c = NULL and the coefficients live in the VECCUDA bv->buffer
   (column j accumulates, column 0 is the scratch c, BV_AddCoefficients_Default, bvimpl.h:306-320).
   Vector variant: h and c are BVOrthogonalizeVec's host arrays, staged through device memory. */
static PetscErrorCode BVGramSchmidt_B200(BV bv, PetscInt j, Vec v, PetscBool *which, PetscScalar *h, PetscScalar *c,
                                         PetscReal *onrm, PetscReal *nrm)
{
  BV_B200     *ctx = (BV_B200 *)bv->data;
  PetscScalar *buf, *pv;
  double       on = 0.0, nr = 0.0;
  PetscInt     jb = v ? bv->k : j;

  PetscFunctionBegin;
  PetscCheck(!bv->matrix && !bv->indef, PetscObjectComm((PetscObject)bv), PETSC_ERR_SUP,
             "BV b200: standard inner product only");
  PetscCall(BVB200Sync(bv));
  if (!v) {
    PetscCall(VecCUDAGetArray(bv->buffer, &buf));
    B200Call(b200_bv_gram_schmidt(ctx->bv, (int)j, NULL, buf + j * (bv->nc + bv->m), buf, onrm ? &on : NULL,
                                  nrm ? &nr : NULL));
    PetscCall(VecCUDARestoreArray(bv->buffer, &buf));
  } else {
    PetscCallCUDA(cudaMemcpy(ctx->stage, h, sizeof(double) * jb, cudaMemcpyHostToDevice));
    PetscCall(VecCUDAGetArray(v, &pv));
    B200Call(b200_bv_gram_schmidt(ctx->bv, 0, pv, ctx->stage, ctx->stage + bv->m + 1, onrm ? &on : NULL,
                                  nrm ? &nr : NULL));
    PetscCall(VecCUDARestoreArray(v, &pv));
    PetscCallCUDA(cudaMemcpy(h, ctx->stage, sizeof(double) * jb, cudaMemcpyDeviceToHost));
    PetscCallCUDA(cudaMemcpy(c, ctx->stage + bv->m + 1, sizeof(double) * (jb + 1), cudaMemcpyDeviceToHost));
  }
  if (onrm) *onrm = on;
  if (nrm) *nrm = nr;
  PetscFunctionReturn(PETSC_SUCCESS);
}

/* BVResize (bvbasic.c:338): new storage through the ABI, the Vec over it rebuilt. */
static PetscErrorCode BVResize_B200(BV bv, PetscInt m, PetscBool copy)
{
  BV_B200 *ctx = (BV_B200 *)bv->data;
  double  *V;

  PetscFunctionBegin;
  B200Call(b200_bv_resize(ctx->bv, (int)m, copy ? 1 : 0));
  PetscCall(VecDestroy(&ctx->v));
  B200Call(b200_bv_get_array(ctx->bv, &V));
  PetscCall(VecCreateSeqCUDAWithArray(PetscObjectComm((PetscObject)bv), 1, m * bv->ld, V, &ctx->v));
  PetscCallCUDA(cudaFree(ctx->stage));
  PetscCallCUDA(cudaMalloc((void **)&ctx->stage, sizeof(double) * 2 * (m + 1)));
  PetscFunctionReturn(PETSC_SUCCESS);
}

/* BVCopy (bvbasic.c:1779): active columns of V into W from W's leading column. */
static PetscErrorCode BVCopy_B200(BV V, BV W)
{
  BV_B200 *v = (BV_B200 *)V->data, *w = (BV_B200 *)W->data;

  PetscFunctionBegin;
  PetscCall(BVB200Sync(V));
  PetscCall(BVB200Sync(W));
  B200Call(b200_bv_copy(v->bv, w->bv));
  PetscFunctionReturn(PETSC_SUCCESS);
}

/* duplicate op (BVDuplicate_Private, bvbasic.c:1619-1632, has already set W's type and sizes):
   carry the orthogonalisation settings into W's device object. */
static PetscErrorCode BVDuplicate_B200(BV V, BV W)
{
  BV_B200 *w = (BV_B200 *)W->data;

  PetscFunctionBegin;
  B200Call(b200_bv_set_orthog_eta(w->bv, V->orthog_eta));
  /* B200_ORTHOG_BLOCK_* number the five BVOrthogBlockType values in the same order */
  B200Call(b200_bv_set_orthog_block(w->bv, (int)V->orthog_block));
  PetscFunctionReturn(PETSC_SUCCESS);
}

/* getmat / restoremat (bvbasic.c:1556, BVRestoreMat_Default :1590): a dense CUDA matrix placed over
   the active columns of the device storage; nothing is copied either way. */
static PetscErrorCode BVGetMat_B200(BV bv, Mat *A)
{
  BV_B200 *ctx = (BV_B200 *)bv->data;
  double  *V;
  PetscInt m = bv->k - bv->l;

  PetscFunctionBegin;
  B200Call(b200_bv_get_array(ctx->bv, &V));
  if (!ctx->Aget) {
    PetscCall(MatCreateDenseCUDA(PetscObjectComm((PetscObject)bv), bv->n, PETSC_DECIDE, bv->N, m, NULL, &ctx->Aget));
    PetscCall(MatDenseSetLDA(ctx->Aget, bv->ld));
  }
  PetscCall(MatDenseCUDAPlaceArray(ctx->Aget, V + (bv->nc + bv->l) * bv->ld));
  *A = ctx->Aget;
  PetscFunctionReturn(PETSC_SUCCESS);
}

static PetscErrorCode BVRestoreMat_B200(BV bv, Mat *A)
{
  BV_B200 *ctx = (BV_B200 *)bv->data;

  PetscFunctionBegin;
  PetscCall(MatDenseCUDAResetArray(ctx->Aget));
  PetscCall(MatDestroy(&ctx->Aget)); /* the active columns may differ at the next getmat */
  *A = NULL;
  PetscFunctionReturn(PETSC_SUCCESS);
}

/* multinplacetrans (BVMultInPlaceHermitianTranspose, bvops.c:268), real scalars. */
static PetscErrorCode BVMultInPlaceTrans_B200(BV V, Mat Q, PetscInt s, PetscInt e)
{
  BV_B200           *ctx = (BV_B200 *)V->data;
  const PetscScalar *q;
  PetscInt           ldq;

  PetscFunctionBegin;
  PetscCall(BVB200Sync(V));
  PetscCall(MatDenseGetLDA(Q, &ldq));
  PetscCall(MatDenseGetArrayRead(Q, &q));
  B200Call(b200_bv_mult_inplace_trans(ctx->bv, q, (int)ldq, (int)s, (int)e));
  PetscCall(MatDenseRestoreArrayRead(Q, &q));
  PetscFunctionReturn(PETSC_SUCCESS);
}

/* normalize (BVNormalize, bvglobal.c:829) for real eigenvectors (eigi null or zero on [l,k)). */
static PetscErrorCode BVNormalize_B200(BV bv, PetscScalar *eigi)
{
  BV_B200 *ctx = (BV_B200 *)bv->data;
  PetscInt i;

  PetscFunctionBegin;
  for (i = bv->l; eigi && i < bv->k; i++)
    PetscCheck(eigi[i] == 0.0, PetscObjectComm((PetscObject)bv), PETSC_ERR_SUP, "BV b200: complex pairs not supported");
  PetscCall(BVB200Sync(bv));
  B200Call(b200_bv_normalize(ctx->bv, NULL));
  PetscFunctionReturn(PETSC_SUCCESS);
}

static PetscErrorCode BVDestroy_B200(BV bv)
{
  BV_B200 *ctx = (BV_B200 *)bv->data;

  PetscFunctionBegin;
  PetscCall(VecDestroy(&ctx->v));
  PetscCall(MatDestroy(&ctx->Aget));
  PetscCallCUDA(cudaFree(ctx->stage));
  PetscCall(VecDestroy(&bv->cv[0]));
  PetscCall(VecDestroy(&bv->cv[1]));
  B200Call(b200_bv_destroy(ctx->bv));
  PetscCall(PetscFree(bv->data));
  bv->cuda = PETSC_FALSE;
  PetscFunctionReturn(PETSC_SUCCESS);
}

PetscErrorCode BVCreate_B200(BV bv)
{
  BV_B200 *ctx;
  PetscInt nloc;
  int      ld;
  double  *V;

  PetscFunctionBegin;
  PetscCheck(bv->nc == 0, PetscObjectComm((PetscObject)bv), PETSC_ERR_SUP, "BV b200: constraints not supported");
  PetscCall(PetscNew(&ctx));
  bv->data = (void *)ctx;
  bv->cuda = PETSC_TRUE; /* columns are VECSEQCUDA, bv->buffer is created with bv->vtype */
  PetscCall(PetscLayoutGetLocalSize(bv->map, &nloc));
  B200Call(b200_bv_create((int)nloc, (int)bv->m, NULL, &ctx->bv));
  B200Call(b200_bv_get_sizes(ctx->bv, NULL, NULL, &ld));
  bv->ld = ld;
  B200Call(b200_bv_get_array(ctx->bv, &V));
  PetscCall(VecCreateSeqCUDAWithArray(PetscObjectComm((PetscObject)bv), 1, bv->m * bv->ld, V, &ctx->v));
  PetscCall(BVCreateVecEmpty(bv, &bv->cv[0]));
  PetscCall(BVCreateVecEmpty(bv, &bv->cv[1]));
  PetscCallCUDA(cudaMalloc((void **)&ctx->stage, sizeof(double) * 2 * (bv->m + 1)));

  bv->ops->mult             = BVMult_B200;
  bv->ops->multvec          = BVMultVec_B200;
  bv->ops->multinplace      = BVMultInPlace_B200;
  bv->ops->dot              = BVDot_B200;
  bv->ops->dotvec           = BVDotVec_B200;
  bv->ops->scale            = BVScale_B200;
  bv->ops->norm             = BVNorm_B200;
  bv->ops->matmult          = BVMatMult_B200;
  bv->ops->copycolumn       = BVCopyColumn_B200;
  bv->ops->getcolumn        = BVGetColumn_B200;
  bv->ops->restorecolumn    = BVRestoreColumn_B200;
  bv->ops->getarray         = BVGetArray_B200;
  bv->ops->restorearray     = BVRestoreArray_B200;
  bv->ops->getarrayread     = BVGetArrayRead_B200;
  bv->ops->restorearrayread = BVRestoreArrayRead_B200;
  bv->ops->gramschmidt      = BVGramSchmidt_B200;
  bv->ops->resize           = BVResize_B200;
  bv->ops->copy             = BVCopy_B200;
  bv->ops->duplicate        = BVDuplicate_B200;
  bv->ops->getmat           = BVGetMat_B200;
  bv->ops->restoremat       = BVRestoreMat_B200;
  bv->ops->multinplacetrans = BVMultInPlaceTrans_B200;
  bv->ops->normalize        = BVNormalize_B200;
  bv->ops->destroy          = BVDestroy_B200;
  PetscFunctionReturn(PETSC_SUCCESS);
}

/* ------------------------------------------------------------------ EPS --- */

typedef struct {
  b200_eps E;
  b200_mat A;   /* borrowed from a b200csr shell, or owned when built from AIJ */
  Mat      own; /* shell created here from an AIJ operator */
  PetscBool mixed; /* -eps_b200_precision mixed: b200_eps_set_precision(B200_PRECISION_MIXED) */
} EPS_B200KS;

static int WhichToB200(EPSWhich w)
{
  switch (w) {
  case EPS_LARGEST_MAGNITUDE:  return B200_LARGEST_MAGNITUDE;
  case EPS_SMALLEST_MAGNITUDE: return B200_SMALLEST_MAGNITUDE;
  case EPS_LARGEST_REAL:       return B200_LARGEST_REAL;
  case EPS_SMALLEST_REAL:      return B200_SMALLEST_REAL;
  default:                     return 0;
  }
}

static PetscErrorCode EPSSetUp_B200KS(EPS eps)
{
  EPS_B200KS *ctx = (EPS_B200KS *)eps->data;
  Mat         A;
  PetscBool   isshift, isaij;
  PetscScalar sigma;

  PetscFunctionBegin;
  PetscCheck(eps->problem_type == EPS_HEP, PetscObjectComm((PetscObject)eps), PETSC_ERR_SUP, "b200ks: EPS_HEP only");
  PetscCall(PetscObjectTypeCompare((PetscObject)eps->st, STSHIFT, &isshift));
  PetscCall(STGetShift(eps->st, &sigma));
  PetscCheck(isshift && sigma == 0.0, PetscObjectComm((PetscObject)eps), PETSC_ERR_SUP, "b200ks: ST shift with sigma=0 only");
  if (!eps->which) PetscCall(EPSSetWhichEigenpairs_Default(eps));
  PetscCheck(WhichToB200(eps->which), PetscObjectComm((PetscObject)eps), PETSC_ERR_SUP, "b200ks: unsupported EPSWhich");
  PetscCheck(!eps->nds, PetscObjectComm((PetscObject)eps), PETSC_ERR_SUP, "b200ks: deflation space not supported");
  PetscCall(EPSSetDimensions_Default(eps, &eps->nev, &eps->ncv, &eps->mpd));
  if (eps->max_it == PETSC_DETERMINE) eps->max_it = PetscMax(100, 2 * eps->n / eps->ncv);
  PetscCall(EPSAllocateSolution(eps, 1));

  PetscCall(STGetMatrix(eps->st, 0, &A));
  PetscCall(MatB200Get(A, &ctx->A));
  if (!ctx->A) {
    PetscCall(PetscObjectTypeCompare((PetscObject)A, MATSEQAIJ, &isaij));
    PetscCheck(isaij, PetscObjectComm((PetscObject)eps), PETSC_ERR_SUP, "b200ks: operator must be MATSEQAIJ or MatCreateB200");
    PetscCall(MatDestroy(&ctx->own));
    PetscCall(MatCreateB200(A, &ctx->own));
    PetscCall(MatB200Get(ctx->own, &ctx->A));
  }
  if (!ctx->E) B200Call(b200_eps_create(NULL, &ctx->E));
  B200Call(b200_eps_set_operators(ctx->E, ctx->A));
  B200Call(b200_eps_set_dimensions(ctx->E, (int)eps->nev, (int)eps->ncv, (int)eps->mpd));
  B200Call(b200_eps_set_tolerances(ctx->E, eps->tol == (PetscReal)PETSC_DETERMINE ? 0.0 : eps->tol, (int)eps->max_it));
  B200Call(b200_eps_set_which_eigenpairs(ctx->E, WhichToB200(eps->which)));
  B200Call(b200_eps_set_precision(ctx->E, ctx->mixed ? B200_PRECISION_MIXED : B200_PRECISION_FP64));
  PetscFunctionReturn(PETSC_SUCCESS);
}

/* -eps_b200_precision fp64|mixed (EPSSetFromOptions calls this, epsopts.c) */
static PetscErrorCode EPSSetFromOptions_B200KS(EPS eps, PetscOptionItems *PetscOptionsObject)
{
  EPS_B200KS *ctx = (EPS_B200KS *)eps->data;
  const char *list[] = {"fp64", "mixed"};
  PetscInt    idx = ctx->mixed ? 1 : 0;
  PetscBool   flg;

  PetscFunctionBegin;
  PetscOptionsHeadBegin(PetscOptionsObject, "EPS b200ks options");
  PetscCall(PetscOptionsEList("-eps_b200_precision", "Arithmetic of the B200 solve", "b200_eps_set_precision", list, 2,
                              list[idx], &idx, &flg));
  if (flg) ctx->mixed = idx == 1 ? PETSC_TRUE : PETSC_FALSE;
  PetscOptionsHeadEnd();
  PetscFunctionReturn(PETSC_SUCCESS);
}

static PetscErrorCode EPSSolve_B200KS(EPS eps)
{
  EPS_B200KS   *ctx = (EPS_B200KS *)eps->data;
  Vec           v0, x;
  PetscScalar  *px;
  const double *d;
  double        lam, err;
  int           nconv, its, reason, i;

  PetscFunctionBegin;
  if (eps->nini) { /* EPSSetUp put the initial vector in column 0 (BVInsertVecs) */
    const PetscScalar *p;
    PetscCall(BVGetColumn(eps->V, 0, &v0));
    PetscCall(VecCUDAGetArrayRead(v0, &p));
    B200Call(b200_eps_set_initial_space_device(ctx->E, p));
    B200Call(b200_eps_solve(ctx->E));
    PetscCall(VecCUDARestoreArrayRead(v0, &p));
    PetscCall(BVRestoreColumn(eps->V, 0, &v0));
  } else B200Call(b200_eps_solve(ctx->E));
  B200Call(b200_eps_get_converged(ctx->E, &nconv));
  B200Call(b200_eps_get_iteration_number(ctx->E, &its));
  B200Call(b200_eps_get_converged_reason(ctx->E, &reason));
  for (i = 0; i < nconv && i < eps->ncv; i++) {
    B200Call(b200_eps_get_eigenpair(ctx->E, i, &lam, NULL));
    B200Call(b200_eps_get_error_estimate(ctx->E, i, &err));
    B200Call(b200_eps_get_eigenvector_device(ctx->E, i, &d));
    eps->eigr[i]   = lam;
    eps->eigi[i]   = 0.0;
    eps->errest[i] = err;
    PetscCall(BVGetColumn(eps->V, i, &x));
    PetscCall(VecCUDAGetArrayWrite(x, &px));
    PetscCallCUDA(cudaMemcpy(px, d, sizeof(double) * eps->nloc, cudaMemcpyDeviceToDevice));
    PetscCall(VecCUDARestoreArrayWrite(x, &px));
    PetscCall(BVRestoreColumn(eps->V, i, &x));
  }
  eps->nconv  = nconv;
  eps->its    = its;
  eps->reason = reason == B200_CONVERGED_TOL ? EPS_CONVERGED_TOL : reason == B200_DIVERGED_ITS ? EPS_DIVERGED_ITS : EPS_DIVERGED_BREAKDOWN;
  PetscFunctionReturn(PETSC_SUCCESS);
}

static PetscErrorCode EPSDestroy_B200KS(EPS eps)
{
  EPS_B200KS *ctx = (EPS_B200KS *)eps->data;

  PetscFunctionBegin;
  if (ctx->E) B200Call(b200_eps_destroy(ctx->E));
  PetscCall(MatDestroy(&ctx->own));
  PetscCall(PetscFree(eps->data));
  PetscFunctionReturn(PETSC_SUCCESS);
}

PetscErrorCode EPSCreate_B200KS(EPS eps)
{
  EPS_B200KS *ctx;

  PetscFunctionBegin;
  PetscCall(PetscNew(&ctx));
  eps->data                = (void *)ctx;
  eps->useds               = PETSC_FALSE;
  eps->categ               = EPS_CATEGORY_KRYLOV;
  eps->ops->setup          = EPSSetUp_B200KS;
  eps->ops->setfromoptions = EPSSetFromOptions_B200KS;
  eps->ops->setupsort      = EPSSetUpSort_Default;
  eps->ops->solve          = EPSSolve_B200KS;
  eps->ops->destroy        = EPSDestroy_B200KS;
  eps->ops->backtransform  = EPSBackTransform_Default;
  eps->ops->computevectors = EPSComputeVectors_Hermitian;
  PetscFunctionReturn(PETSC_SUCCESS);
}

/* Register both types (call once after SlepcInitialize). */
PetscErrorCode SlepcB200Register(void)
{
  PetscFunctionBegin;
  PetscCall(BVRegister("b200", BVCreate_B200));
  PetscCall(EPSRegister("b200ks", EPSCreate_B200KS));
  PetscFunctionReturn(PETSC_SUCCESS);
}
