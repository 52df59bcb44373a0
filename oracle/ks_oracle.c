/*
 * ks_oracle.c -- CPU oracle for the Hermitian Krylov-Schur inner loop.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker that the GPU library is
 * compared against; it is never linked into the product library.  Only the
 * tests, the smoke check and the CPU-baseline leg of the benchmark load it.
 *
 * It restates, in plain C on the host, the arithmetic of the SLEPc 3.22 path
 *
 *   EPSSolve -> EPSSolve_KrylovSchur_Default -> BVMatLanczos ->
 *   BVOrthonormalizeColumn (CGS + DGKS "if needed") -> DSSolve_HEP_QR ->
 *   DSSort -> DSUpdateExtraRow -> EPSKrylovConvergence -> DSTruncate ->
 *   BVMultInPlace -> BVCopyColumn
 *
 * with the same order of operations, the same BLAS/LAPACK calls (dgemv,
 * dgemm, dlartg, drot, dsteqr, dsytrd, dorgtr from the OpenBLAS that ships
 * with scipy) and the same default parameters.  Each function names the
 * reference lines it follows (paths relative to the SLEPc source tree).
 *
 * Deliberate difference: PETSc's random number generator (used by
 * BVSetRandomColumn after a Lanczos breakdown) is not part of the SLEPc
 * tree, so a counter-based splitmix64 uniform [0,1) generator stands in for
 * it.  The initial vector is always supplied by the caller
 * (EPSSetInitialSpace semantics, src/eps/interface/epssolve.c:852).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ---- BLAS / LAPACK from scipy's bundled OpenBLAS (exported with a scipy_ prefix) ---- */
extern void scipy_dgemv_(const char *, const int *, const int *, const double *, const double *,
                         const int *, const double *, const int *, const double *, double *, const int *,
                         size_t);
extern void scipy_dgemm_(const char *, const char *, const int *, const int *, const int *, const double *,
                         const double *, const int *, const double *, const int *, const double *, double *,
                         const int *, size_t, size_t);
extern void scipy_dlartg_(const double *, const double *, double *, double *, double *);
extern void scipy_drot_(const int *, double *, const int *, double *, const int *, const double *,
                        const double *);
extern void scipy_dsteqr_(const char *, const int *, double *, double *, double *, const int *, double *,
                          int *, size_t);
extern void scipy_dsytrd_(const char *, const int *, double *, const int *, double *, double *, double *,
                          double *, const int *, int *, size_t);
extern void scipy_dorgtr_(const char *, const int *, double *, const int *, const double *, double *,
                          const int *, int *, size_t);
extern void scipy_openblas_set_num_threads(int);

#define ORC_MACHINE_EPS DBL_EPSILON

/* status codes (mirroring the product's b200_status numbering) */
enum { ORC_OK = 0, ORC_ERR_ARG = 1, ORC_ERR_LAPACK = 3, ORC_ERR_INNER = 4, ORC_ERR_BREAKDOWN = 5 };

/* sorting criteria, src/sys/slepcsc.c:152-210 */
enum { ORC_LARGEST_MAGNITUDE = 1, ORC_SMALLEST_MAGNITUDE = 2, ORC_LARGEST_REAL = 3, ORC_SMALLEST_REAL = 4 };

/* converged reasons, include/slepceps.h (EPSConvergedReason) */
enum { ORC_CONVERGED_TOL = 1, ORC_DIVERGED_ITS = -1, ORC_DIVERGED_BREAKDOWN = -2, ORC_ITERATING = 0 };

void oracle_set_threads(int nthreads)
{
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
  if (nthreads > 0) scipy_openblas_set_num_threads(nthreads);
}

/* ======================================================================
 * CSR sparse matrix-vector product y = A x (PETSc MatMult_SeqAIJ semantics:
 * each row summed in index order).
 * ====================================================================== */
void oracle_spmv(int n, const int *rowptr, const int *colind, const double *vals, const double *x, double *y)
{
  int i;
#pragma omp parallel for schedule(static)
  for (i = 0; i < n; i++) {
    double s = 0.0;
    for (int p = rowptr[i]; p < rowptr[i + 1]; p++) s += vals[p] * x[colind[p]];
    y[i] = s;
  }
}

/* CSR with the same row-order sums for a rectangular matrix (rows x any) */
static void csr_mult(int rows, const int *rowptr, const int *colind, const double *vals, const double *x, double *y)
{
  oracle_spmv(rows, rowptr, colind, vals, x, y);
}

/*
 * Explicit transpose, MatTranspose_SeqAIJ semantics: row c of A^T lists the
 * rows i of A with a nonzero in column c in ascending i, so its sum runs in
 * that order.  rowptr_t has cols+1 entries; colind_t / vals_t have nnz.
 */
void oracle_csr_transpose(int rows, int cols, const int *rowptr, const int *colind, const double *vals,
                          int *rowptr_t, int *colind_t, double *vals_t)
{
  int i, c, p;
  int *next = (int *)malloc(sizeof(int) * ((size_t)cols + 1));
  for (c = 0; c <= cols; c++) rowptr_t[c] = 0;
  for (p = 0; p < rowptr[rows]; p++) rowptr_t[colind[p] + 1]++;
  for (c = 0; c < cols; c++) rowptr_t[c + 1] += rowptr_t[c];
  for (c = 0; c < cols; c++) next[c] = rowptr_t[c];
  for (i = 0; i < rows; i++)
    for (p = rowptr[i]; p < rowptr[i + 1]; p++) {
      int q = next[colind[p]]++;
      colind_t[q] = i;
      vals_t[q] = vals[p];
    }
  free(next);
}

/*
 * The operator of the eigensolver: a square CSR matrix, or the shell
 * C = A^T A of the SVD cross solver, applied as w = A x then y = A^T w
 * (MatMult_Cross, src/svd/impls/cross/cross.c:31-41, explicit transpose as
 * SVDSetUp builds by default, src/svd/interface/svdsetup.c:300-305).
 */
typedef struct {
  int n;                    /* operator dimension */
  int cross;                /* 0: y = A x (A n x n); 1: y = A^T (A x) (A m x n) */
  int m;                    /* rows of A (cross) */
  const int *rp, *ci;       /* A */
  const double *va;
  const int *rpt, *cit;     /* A^T (cross) */
  const double *vat;
  double *w;                /* m entries (cross) */
} orc_op;

static void op_apply(const orc_op *op, const double *x, double *y)
{
  if (!op->cross) {
    oracle_spmv(op->n, op->rp, op->ci, op->va, x, y);
    return;
  }
  csr_mult(op->m, op->rp, op->ci, op->va, x, op->w);
  csr_mult(op->n, op->rpt, op->cit, op->vat, op->w, y);
}

static double nrm2(int n, const double *x)
{
  /* plain two-norm; PETSc VecNorm(NORM_2) -> BLASnrm2 */
  double s = 0.0;
  int i;
#pragma omp parallel for reduction(+ : s) schedule(static)
  for (i = 0; i < n; i++) s += x[i] * x[i];
  return sqrt(s);
}

/* counter-based uniform [0,1) generator standing in for PETSc's VecSetRandom */
static uint64_t splitmix64(uint64_t z)
{
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}
double oracle_random_entry(uint64_t seed, uint64_t stream, uint64_t i)
{
  uint64_t z = splitmix64(seed ^ splitmix64(stream * 0x100000001B3ULL + i));
  return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

/* ======================================================================
 * BV: column-major basis V (n rows, m columns, leading dimension ld) plus
 * the coefficient buffer of BVGetBufferVec (m x m, column j holds the
 * Gram-Schmidt coefficients of column j; column 0 doubles as scratch),
 * src/sys/classes/bv/interface/bvbasic.c:775-790.  No constraints (nc=0).
 * ====================================================================== */
typedef struct {
  int n, m, ld;
  double *V;
  double *buf;     /* m*m */
  double *hvec;    /* scratch for the vector variant */
  double *cvec;
  double eta;      /* orthog_eta, bvfunc.c:178 */
  double deftol;   /* 10*eps, bvfunc.c:184 */
  uint64_t seed;
  uint64_t nrand;  /* number of random columns generated so far */
} obv;

/* BV_SafeSqrt, include/slepc/private/bvimpl.h:121-141 (definite inner product) */
static int safe_sqrt(const obv *bv, double alpha, double *res)
{
  if (!(alpha > -bv->deftol)) return ORC_ERR_INNER;
  *res = (alpha < 0.0) ? 0.0 : sqrt(alpha);
  return ORC_OK;
}

/* BVDotVec_BLAS_Private (bvblas.c:240-261): q = V(:,0:k)^T y via gemv "C" */
static void bv_dotvec(const obv *bv, int k, const double *y, double *q)
{
  const double one = 1.0, zero = 0.0;
  const int inc = 1;
  if (k <= 0) return;
  scipy_dgemv_("C", &bv->n, &k, &one, bv->V, &bv->ld, y, &inc, &zero, q, &inc, 1);
}

/* BVMultVec_BLAS_Private (bvblas.c:50-66): y = beta*y + alpha*V(:,0:k) q */
static void bv_multvec(const obv *bv, int k, double alpha, const double *q, double beta, double *y)
{
  const int inc = 1;
  if (k <= 0) return;
  scipy_dgemv_("N", &bv->n, &k, &alpha, bv->V, &bv->ld, q, &inc, &beta, y, &inc, 1);
}

/*
 * BVOrthogonalizeCGS1, bvorthog.c:91-132, for a column (v == NULL) or for an
 * external vector.  j = number of columns to orthogonalize against (the
 * column index itself in the column case).  c receives the new coefficients,
 * h accumulates them (BV_AddCoefficients, bvimpl.h:308-325).
 */
static int cgs1(obv *bv, int j, double *v, double *h, double *c, double *onorm, double *norm)
{
  double beta = 0.0, sum;
  int i, st;
  int col = (v == NULL);
  double *w = col ? bv->V + (size_t)j * bv->ld : v;

  if (onorm || norm) {
    if (col) {
      /* BVDotColumnInc (bvorthog.c:32-47): includes column j against itself */
      bv_dotvec(bv, j + 1, w, c);
      if ((st = safe_sqrt(bv, c[j], &beta))) return st;  /* BV_SquareRoot */
    } else {
      bv_dotvec(bv, j, w, c);
      beta = nrm2(bv->n, w);                                /* BVNormVec */
    }
  } else {
    bv_dotvec(bv, j, w, c);
  }
  /* q = v - V h (BVMultColumn / BVMultVec) */
  bv_multvec(bv, j, -1.0, c, 1.0, w);
  if (onorm) *onorm = beta;
  if (norm) {
    /* estimate |v'| from |v| (bvorthog.c:124-127) */
    sum = 0.0;
    for (i = 0; i < j; i++) sum += c[i] * c[i];                  /* BV_SquareSum */
    *norm = beta * beta - sum;
    if (*norm <= 0.0) *norm = nrm2(bv->n, w);
    else *norm = sqrt(*norm);
  }
  for (i = 0; i < j; i++) h[i] += c[i];                         /* BV_AddCoefficients */
  return ORC_OK;
}

/*
 * BVOrthogonalizeGS with BV_ORTHOG_CGS and BV_ORTHOG_REFINE_IFNEEDED,
 * bvorthog.c:145-217.  Returns the final norm and the lindep flag; in the
 * column case stores the norm next to the coefficients (bvorthog.c:209-214).
 */
static int orthogonalize_gs(obv *bv, int j, double *v, double *norm, int *lindep)
{
  double *h, *c, onrm = 0.0, nrm = 0.0;
  int l, st, i;
  if (v) { h = bv->hvec; c = bv->cvec; }
  else { h = bv->buf + (size_t)j * bv->m; c = bv->buf; /* column 0 = scratch */ }
  for (i = 0; i < j; i++) h[i] = 0.0;                          /* BV_CleanCoefficients */
  if ((st = cgs1(bv, j, v, h, c, &onrm, &nrm))) return st;
  l = 1;
  while (l < 3 && nrm != 0.0 && fabs(nrm) < bv->eta * fabs(onrm)) {
    l++;
    if ((st = cgs1(bv, j, v, h, c, &onrm, &nrm))) return st;
  }
  *lindep = !(nrm != 0.0 && fabs(nrm) >= bv->eta * fabs(onrm));
  if (norm) {
    *norm = nrm;
    if (!v) h[j] = (*lindep) ? 0.0 : nrm;                       /* BV_SetValue(bv,k,k,h,...) */
  }
  return ORC_OK;
}

/* BVSetRandomColumn stand-in (bvops.c:360-379) */
static void set_random_column(obv *bv, int j)
{
  double *w = bv->V + (size_t)j * bv->ld;
  uint64_t stream = bv->nrand++;
  for (int i = 0; i < bv->n; i++) w[i] = oracle_random_entry(bv->seed, stream, (uint64_t)i);
}

static void scale_column(obv *bv, int j, double alpha)
{
  double *w = bv->V + (size_t)j * bv->ld;
  int i;
  if (alpha == 1.0) return;
#pragma omp parallel for schedule(static)
  for (i = 0; i < bv->n; i++) w[i] *= alpha;
}

/* BVOrthonormalizeColumn, bvorthog.c:380-427 (replace = FALSE) */
static int orthonormalize_column(obv *bv, int j, double *norm, int *lindep)
{
  double nrm;
  int lnd, st;
  if ((st = orthogonalize_gs(bv, j, NULL, &nrm, &lnd))) return st;
  if (nrm != 1.0 && nrm != 0.0) scale_column(bv, j, 1.0 / nrm);
  if (norm) *norm = nrm;
  if (lindep) *lindep = lnd;
  return ORC_OK;
}

/* ======================================================================
 * DS of type HEP, compact (arrowhead + tridiagonal) storage.
 * T holds d (diagonal) at T[0..ld) and e (off-diagonal/arrow) at T[ld..2ld);
 * Q is ld x ld column-major.  src/sys/classes/ds/impls/hep/dshep.c
 * ====================================================================== */
typedef struct {
  int ld, n, l, k, t;
  int state;     /* 0 RAW, 1 INTERMEDIATE, 2 CONDENSED, 3 TRUNCATED */
  double *d, *e, *Q, *rwork;
  int *perm;
  int which;
} ods;

/* DSSetIdentity, dspriv.c:407-426: zero columns l..n-1, unit diagonal */
static void ds_set_identity(ods *ds)
{
  memset(ds->Q + (size_t)ds->l * ds->ld, 0, sizeof(double) * (size_t)ds->ld * (ds->n - ds->l));
  for (int i = ds->l; i < ds->n; i++) ds->Q[i + (size_t)i * ds->ld] = 1.0;
}

/* DSArrowTridiag, dshep.c:221-265 (Rutishauser's reduction of an arrowhead) */
static void ds_arrow_tridiag(int n, double *d, double *e, double *Q, int ld)
{
  int i, j, j2;
  const int one = 1;
  double c, s, p, off, temp;
  if (n <= 2) return;
  for (j = 0; j < n - 2; j++) {
    temp = e[j + 1];
    scipy_dlartg_(&temp, &e[j], &c, &s, &e[j + 1]);
    s = -s;
    temp = d[j + 1];
    e[j] = c * s * (temp - d[j]);
    d[j + 1] = s * s * d[j] + c * c * temp;
    d[j] = c * c * d[j] + s * s * temp;
    j2 = j + 2;
    scipy_drot_(&j2, Q + (size_t)j * ld, &one, Q + (size_t)(j + 1) * ld, &one, &c, &s);
    for (i = j - 1; i >= 0; i--) {
      off = -s * e[i];
      e[i] = c * e[i];
      temp = e[i + 1];
      scipy_dlartg_(&temp, &off, &c, &s, &e[i + 1]);
      s = -s;
      temp = (d[i] - d[i + 1]) * s - 2.0 * c * e[i];
      p = s * temp;
      d[i + 1] += p;
      d[i] -= p;
      e[i] = -e[i] - c * temp;
      scipy_drot_(&j2, Q + (size_t)i * ld, &one, Q + (size_t)(i + 1) * ld, &one, &c, &s);
    }
  }
}

/* SlepcCompare* comparators, src/sys/slepcsc.c:152-210 (real case) */
static int sc_compare(int which, double a, double b)
{
  double x, y;
  switch (which) {
  case ORC_LARGEST_MAGNITUDE: x = fabs(a); y = fabs(b); return (x < y) ? 1 : (x > y) ? -1 : 0;
  case ORC_SMALLEST_MAGNITUDE: x = fabs(a); y = fabs(b); return (x > y) ? 1 : (x < y) ? -1 : 0;
  case ORC_LARGEST_REAL: return (a < b) ? 1 : (a > b) ? -1 : 0;
  case ORC_SMALLEST_REAL: return (a > b) ? 1 : (a < b) ? -1 : 0;
  default: return 0;
  }
}

/* DSSolve_HEP_QR (compact), dshep.c:383-427 with DSIntermediate_HEP :267-321 */
static int ds_solve_hep_qr(ods *ds, double *wr)
{
  int i, info = 0, n1, ld = ds->ld, l = ds->l, n = ds->n;
  size_t off = (size_t)l + (size_t)l * ld;
  int na = ds->k - l + 1;
  if (na < 0) na = 0;
  ds_set_identity(ds);
  if (ds->state < 1) ds_arrow_tridiag(na, ds->d + l, ds->e + l, ds->Q + off, ld);
  for (i = 0; i < l; i++) wr[i] = ds->d[i];
  n1 = n - l;
  if (n1 > 0) scipy_dsteqr_("V", &n1, ds->d + l, ds->e + l, ds->Q + off, &ld, ds->rwork, &info, 1);
  if (info) return ORC_ERR_LAPACK;
  for (i = l; i < n; i++) wr[i] = ds->d[i];
  if (n > 1) memset(ds->e, 0, sizeof(double) * (size_t)(n - 1));
  ds->state = 2;
  return ORC_OK;
}

/* DSSortEigenvaluesReal_Private (dspriv.c:254-273) + DSPermuteColumns_Private (:279-301) + DSSort_HEP (dshep.c:323-347) */
static void ds_sort_hep(ods *ds, double *wr)
{
  int i, j, tmp, result, l = ds->l, n = ds->n, ld = ds->ld, p, k;
  int *perm = ds->perm;
  double re, rtmp;
  for (i = 0; i < n; i++) perm[i] = i;
  for (i = l + 1; i < ds->t; i++) {
    re = ds->d[perm[i]];
    j = i - 1;
    result = sc_compare(ds->which, re, ds->d[perm[j]]);
    while (result < 0 && j >= l) {
      tmp = perm[j]; perm[j] = perm[j + 1]; perm[j + 1] = tmp; j--;
      if (j >= l) result = sc_compare(ds->which, re, ds->d[perm[j]]);
    }
  }
  for (i = l; i < n; i++) wr[i] = ds->d[perm[i]];
  for (i = l; i < n; i++) {
    p = perm[i];
    if (p != i) {
      j = i + 1;
      while (perm[j] != i) j++;
      perm[j] = p; perm[i] = i;
      for (k = 0; k < n; k++) {
        rtmp = ds->Q[k + (size_t)p * ld]; ds->Q[k + (size_t)p * ld] = ds->Q[k + (size_t)i * ld]; ds->Q[k + (size_t)i * ld] = rtmp;
      }
    }
  }
  for (i = l; i < n; i++) ds->d[i] = wr[i];
}

/* DSUpdateExtraRow_HEP (compact), dshep.c:349-381 */
static void ds_update_extra_row(ods *ds)
{
  int n = ds->n, ld = ds->ld;
  double beta = ds->e[n - 1];
  for (int i = 0; i < n; i++) ds->e[i] = beta * ds->Q[n - 1 + (size_t)i * ld];
  ds->k = n;
}

/* DSTruncate_HEP (compact, trim = FALSE), dshep.c:643-671 */
static void ds_truncate(ods *ds, int n)
{
  ds->k = n;        /* extra row present */
  ds->t = ds->n;
  ds->n = n;
  ds->state = 3;
}

/* ======================================================================
 * EPS Krylov-Schur (Hermitian, Ritz extraction, locking) solve.
 * ====================================================================== */
typedef struct {
  int nconv, its, reason;
  long lanczos_steps;   /* total number of SpMV+orthonormalization steps */
  long gs_passes;       /* total number of CGS passes (DGKS refinements included) */
  long column_visits;   /* sum over Lanczos steps j of (j+2): basis columns one CGS pass reads */
  int restarts_done;
} orc_info;

/* EPSGetStartVector, epssolve.c:841-870 (i > 0 uses a random vector) */
static int get_start_vector(obv *bv, int i, int nini, int *breakdown)
{
  double norm;
  int lindep, st;
  if (i > 0 || nini == 0) set_random_column(bv, i);   /* epssolve.c:852 */
  if ((st = orthogonalize_gs(bv, i, NULL, &norm, &lindep))) return st;
  if (breakdown) *breakdown = lindep;
  else if (lindep || norm == 0.0) return ORC_ERR_BREAKDOWN;
  scale_column(bv, i, 1.0 / norm);
  return ORC_OK;
}

/*
 * oracle_eps_solve: EPSSolve (epssolve.c:119-229) on a Hermitian CSR matrix
 * with EPSKRYLOVSCHUR defaults.
 *   which    : ORC_LARGEST_MAGNITUDE ... ORC_SMALLEST_REAL
 *   v0       : initial vector (EPSSetInitialSpace with one vector)
 *   ncv, mpd : subspace dimensions (mpd <= 0 means mpd = ncv)
 *   max_it   : <= 0 means max(100, 2n/ncv), krylovschur.c:113
 *   max_restarts : > 0 stops after that many restarts (bounded CPU sample;
 *                  reason stays ITERATING); 0 = run to completion
 * Outputs: eigr[ncv+1] and errest[ncv+1] in the solver's internal order,
 * X (n x nconv, ld = n) the converged Ritz vectors sorted by SlepcSortEigenvalues,
 * evals (nconv) sorted values; info.
 */
/* EPSKrylovSchurSetLocking (krylovschur.c:427-434): 1 (default) locks converged pairs at a restart;
   0 selects the non-locking variant (krylovschur.c:295), which keeps them in the active subspace. */
static int g_ks_lock = 1;
void oracle_set_locking(int lock) { g_ks_lock = lock ? 1 : 0; }

static int eps_solve_op(const orc_op *op, const double *v0, int nev, int ncv, int mpd, double tol, int max_it,
                        int which, int max_restarts, double *evals, double *X, double *errest_out, int *info_out)
{
  const int n = op->n;
  obv bv;
  ods ds;
  orc_info info;
  int st = ORC_OK, i, j, k, l, nv, breakdown = 0, lindep, m, nconv_loc;
  double beta = 0.0, norm, *eigr, *errest;
  int *perm;
  const double keep = 0.5;

  memset(&info, 0, sizeof(info));
  if (n <= 0 || nev <= 0 || ncv <= nev || ncv > n) return ORC_ERR_ARG;
  if (mpd <= 0) mpd = ncv;
  if (max_it <= 0) max_it = (2 * n / ncv > 100) ? 2 * n / ncv : 100;

  bv.n = n; bv.m = ncv + 1; bv.ld = n;
  bv.V = (double *)calloc((size_t)bv.ld * bv.m, sizeof(double));
  bv.buf = (double *)calloc((size_t)bv.m * bv.m, sizeof(double));
  bv.hvec = (double *)calloc(bv.m, sizeof(double));
  bv.cvec = (double *)calloc(bv.m, sizeof(double));
  bv.eta = 0.7071; bv.deftol = 10 * ORC_MACHINE_EPS; bv.seed = 0x5eedULL; bv.nrand = 0;

  ds.ld = ncv + 1; ds.n = 0; ds.l = 0; ds.k = 0; ds.t = 0; ds.state = 0; ds.which = which;
  ds.d = (double *)calloc((size_t)3 * ds.ld, sizeof(double));
  ds.e = ds.d + ds.ld;
  ds.Q = (double *)calloc((size_t)ds.ld * ds.ld, sizeof(double));
  ds.rwork = (double *)calloc((size_t)2 * ds.ld + 2, sizeof(double));
  ds.perm = (int *)calloc(ds.ld, sizeof(int));
  eigr = (double *)calloc(ds.ld, sizeof(double));
  errest = (double *)calloc(ds.ld, sizeof(double));
  perm = (int *)calloc(ds.ld, sizeof(int));

  /* EPSSetUp: BVInsertVecs(V,0,&k,IS,TRUE) (epssetup.c:421-427, bvfunc.c:331-374): a zero or
   * dependent initial vector is dropped and the start vector is then random */
  {
    int nini = 0;
    if (v0) {
      memcpy(bv.V, v0, sizeof(double) * (size_t)n);
      if ((st = orthogonalize_gs(&bv, 0, NULL, &norm, &lindep))) goto done;
      if (!(norm == 0.0 || lindep)) { scale_column(&bv, 0, 1.0 / norm); nini = 1; }
    }
    /* EPSGetStartVector(eps,0,NULL) */
    if ((st = get_start_vector(&bv, 0, nini, NULL))) goto done;
  }

  l = 0;
  info.reason = ORC_ITERATING;
  while (info.reason == ORC_ITERATING) {
    info.its++;
    nv = (info.nconv + mpd < ncv) ? info.nconv + mpd : ncv;
    /* DSSetDimensions(ds,nv,nconv,nconv+l) */
    ds.n = nv; ds.t = nv; ds.l = info.nconv; ds.k = info.nconv + l;
    /* BVMatLanczos(V,Op,T,nconv+l,&nv,&beta,&breakdown), bvkrylov.c:165-226 */
    k = info.nconv + l;
    m = nv;
    breakdown = 0;
    for (j = k; j < m; j++) {
      op_apply(op, bv.V + (size_t)j * bv.ld, bv.V + (size_t)(j + 1) * bv.ld);
      if ((st = orthonormalize_column(&bv, j + 1, &beta, &lindep))) goto done;
      info.lanczos_steps++;
      info.column_visits += j + 2;
      if (lindep) { m = j + 1; breakdown = 1; break; }
    }
    for (j = k; j < m; j++) {
      ds.d[j] = bv.buf[j + (size_t)(j + 1) * bv.m];      /* alpha_j */
      ds.e[j] = bv.buf[j + 1 + (size_t)(j + 1) * bv.m];  /* beta_j */
    }
    nv = m;
    ds.n = nv; ds.t = nv; ds.l = info.nconv; ds.k = info.nconv + l;
    ds.state = l ? 0 : 1;                                 /* RAW : INTERMEDIATE */

    /* DSSolve + DSSort + DSUpdateExtraRow */
    if ((st = ds_solve_hep_qr(&ds, eigr))) goto done;
    ds_sort_hep(&ds, eigr);
    ds_update_extra_row(&ds);

    /* EPSKrylovConvergence (epskrylov.c:207-295), EPSConvergedRelative (epsdefault.c:224-232) */
    {
      int marker = -1, kk;
      for (kk = info.nconv; kk < nv; kk++) {
        double re = eigr[kk];
        double resnorm = fabs(ds.Q[ds.n - 1 + (size_t)kk * ds.ld]) * beta * 1.0;
        double wabs = fabs(re);
        errest[kk] = (wabs != 0.0) ? resnorm / wabs : DBL_MAX;
        if (marker == -1 && errest[kk] >= tol) marker = kk;
        if (marker != -1) break;
      }
      if (marker != -1) kk = marker;
      k = kk;
    }
    /* EPSStoppingBasic, epsdefault.c:290-305 */
    if (k >= nev) info.reason = ORC_CONVERGED_TOL;
    else if (info.its >= max_it) info.reason = ORC_DIVERGED_ITS;
    nconv_loc = k;
    (void)nconv_loc;

    /* update l (krylovschur.c:290-296) */
    if (info.reason != ORC_ITERATING || breakdown || k == nv) l = 0;
    else {
      l = (int)((nv - k) * keep);
      if (l < 1) l = 1;
    }
    if (!g_ks_lock && l > 0) { /* non-locking variant: reset the number of converged pairs */
      l += k;
      k = 0;
    }

    if (info.reason == ORC_ITERATING) {
      if (breakdown || k == nv) {
        if (k < nev) {
          int bd = 0;
          if ((st = get_start_vector(&bv, k, 1, &bd))) goto done;
          if (bd) info.reason = ORC_DIVERGED_BREAKDOWN;
        }
      } else {
        ds_truncate(&ds, k + l);
      }
    }
    /* BVMultInPlace(V,Q,nconv,k+l) with active columns [nconv,nv) (bvblas.c:74-106, 64-row blocks) */
    {
      int s = info.nconv, e = k + l, ncols = e - s, kq = nv - info.nconv, bs = 64, rr;
      const double one = 1.0, zero = 0.0;
      if (ncols > 0 && kq > 0) {
        double *work = (double *)malloc(sizeof(double) * (size_t)bs * ncols);
        const double *pb = ds.Q + (size_t)info.nconv + (size_t)s * ds.ld;
        double *A = bv.V + (size_t)info.nconv * bv.ld;
        int r0 = n % bs;
        if (r0) {
          scipy_dgemm_("N", "N", &r0, &ncols, &kq, &one, A, &bv.ld, pb, &ds.ld, &zero, work, &r0, 1, 1);
          for (j = 0; j < ncols; j++) memcpy(bv.V + (size_t)(s + j) * bv.ld, work + (size_t)j * r0, sizeof(double) * r0);
        }
        for (rr = r0; rr < n; rr += bs) {
          scipy_dgemm_("N", "N", &bs, &ncols, &kq, &one, A + rr, &bv.ld, pb, &ds.ld, &zero, work, &bs, 1, 1);
          for (j = 0; j < ncols; j++) memcpy(bv.V + (size_t)(s + j) * bv.ld + rr, work + (size_t)j * bs, sizeof(double) * bs);
        }
        free(work);
      }
    }
    if (info.reason == ORC_ITERATING && !breakdown) {
      /* BVCopyColumn(V,nv,k+l) */
      memcpy(bv.V + (size_t)(k + l) * bv.ld, bv.V + (size_t)nv * bv.ld, sizeof(double) * (size_t)n);
    }
    info.nconv = k;
    info.restarts_done++;
    if (max_restarts > 0 && info.restarts_done >= max_restarts && info.reason == ORC_ITERATING) break;
  }

  /* EPSSolve post-processing: SlepcSortEigenvalues (slepcsc.c:89-149, real case) */
  for (i = 0; i < ncv; i++) perm[i] = i;
  for (i = info.nconv - 1; i >= 0; i--) {
    double re = eigr[perm[i]];
    j = i + 1;
    while (j < info.nconv) {
      if (sc_compare(which, re, eigr[perm[j]]) <= 0) break;
      int tmp = perm[j - 1]; perm[j - 1] = perm[j]; perm[j] = tmp;
      j++;
    }
  }
  for (i = 0; i < info.nconv; i++) {
    if (evals) evals[i] = eigr[perm[i]];
    if (errest_out) errest_out[i] = errest[perm[i]];
    if (X) memcpy(X + (size_t)i * n, bv.V + (size_t)perm[i] * bv.ld, sizeof(double) * (size_t)n);
  }

done:
  if (info_out) {
    info_out[0] = info.nconv;
    info_out[1] = info.its;
    info_out[2] = info.reason;
    info_out[3] = (int)info.lanczos_steps;
    info_out[4] = info.restarts_done;
    info_out[5] = (int)info.column_visits;
  }
  free(bv.V); free(bv.buf); free(bv.hvec); free(bv.cvec);
  free(ds.d); free(ds.Q); free(ds.rwork); free(ds.perm);
  free(eigr); free(errest); free(perm);
  return st;
}

int oracle_eps_solve(int n, const int *rowptr, const int *colind, const double *vals, const double *v0,
                     int nev, int ncv, int mpd, double tol, int max_it, int which, int max_restarts,
                     double *evals, double *X, double *errest_out, int *info_out)
{
  orc_op op;
  memset(&op, 0, sizeof(op));
  op.n = n; op.rp = rowptr; op.ci = colind; op.va = vals;
  return eps_solve_op(&op, v0, nev, ncv, mpd, tol, max_it, which, max_restarts, evals, X, errest_out, info_out);
}

/*
 * oracle_svd_cross: SVDSolve with SVDCROSS for a standard problem whose
 * matrix A (m x n, m >= n; a caller with m < n passes the transpose, as
 * SVDSetUp swaps A and A^T, svdsetup.c:300-314) is given with its explicit
 * transpose.  Follows
 *   SVDSetUp_Cross (cross.c:160-250): EPS_HEP on C = A^T A, which =
 *     largest (smallest) magnitude for the largest (smallest) triplets,
 *     EPS tol = svd tol (1e-9 = SLEPC_DEFAULT_TOL/10 when tol <= 0);
 *   SVDSolve_Cross (cross.c:256-285): sigma_i = sqrt(lambda_i), a negative
 *     lambda > -10 eps reset to 0, below that an error;
 *   SVDSolve's sort (svdsolve.c): ascending sort, reversed for the largest;
 *   SVDComputeVectors_Cross + SVDComputeVectors_Left (cross.c:346-352,
 *     svdsolve.c:21-75): V_i = eigenvector i, U = A V, BVOrthogonalize(U)
 *     by Gram-Schmidt column after column (bvorthog.c:507-548);
 *   SVDComputeError (svdsolve.c:485-580) relative: sqrt(n1^2 + n2^2) /
 *     (sigma sqrt(2)), n1 = ||A v - sigma u||, n2 = ||A^T u - sigma v||.
 * which_svd: 0 largest, 1 smallest.  Outputs (in SVD order, nconv entries):
 * sigma, U (m x nconv), V (n x nconv), rel_error; info as oracle_eps_solve.
 */
int oracle_svd_cross(int m, int n, const int *rowptr, const int *colind, const double *vals, const int *rowptr_t,
                     const int *colind_t, const double *vals_t, const double *v0, int nsv, int ncv, int mpd,
                     double tol, int max_it, int which_svd, int max_restarts, double *sigma_out, double *U_out,
                     double *V_out, double *rel_error, int *info_out)
{
  orc_op op;
  obv bu;
  int st, i, j, nconv, lindep, *perm;
  double *lam, *X, *sig, norm;
  if (m < n || n <= 0) return ORC_ERR_ARG;
  memset(&op, 0, sizeof(op));
  op.n = n; op.cross = 1; op.m = m;
  op.rp = rowptr; op.ci = colind; op.va = vals;
  op.rpt = rowptr_t; op.cit = colind_t; op.vat = vals_t;
  op.w = (double *)malloc(sizeof(double) * (size_t)m);
  lam = (double *)calloc((size_t)ncv + 1, sizeof(double));
  sig = (double *)calloc((size_t)ncv + 1, sizeof(double));
  perm = (int *)calloc((size_t)ncv + 1, sizeof(int));
  X = (double *)calloc((size_t)n * (ncv + 1), sizeof(double));
  if (tol <= 0.0) tol = 1e-9;
  st = eps_solve_op(&op, v0, nsv, ncv, mpd, tol, max_it,
                    which_svd == 0 ? ORC_LARGEST_MAGNITUDE : ORC_SMALLEST_MAGNITUDE, max_restarts, lam, X, NULL,
                    info_out);
  if (st) goto done;
  nconv = info_out ? info_out[0] : 0;
  for (i = 0; i < nconv; i++) {
    double s = lam[i];
    if (s <= -10 * ORC_MACHINE_EPS) { st = ORC_ERR_ARG; goto done; }
    if (s < 0.0) s = 0.0;
    sig[i] = sqrt(s);
  }
  /* sort: insertion sort ascending (stable), reversed for the largest */
  for (i = 0; i < nconv; i++) perm[i] = i;
  for (i = 1; i < nconv; i++) {
    int t = perm[i];
    j = i - 1;
    while (j >= 0 && sig[perm[j]] > sig[t]) { perm[j + 1] = perm[j]; j--; }
    perm[j + 1] = t;
  }
  if (which_svd == 0)
    for (i = 0; i < nconv / 2; i++) { int t = perm[i]; perm[i] = perm[nconv - 1 - i]; perm[nconv - 1 - i] = t; }

  /* U = A V, then Gram-Schmidt over the columns in order */
  bu.n = m; bu.m = nconv > 0 ? nconv : 1; bu.ld = m;
  bu.V = (double *)calloc((size_t)m * bu.m, sizeof(double));
  bu.buf = (double *)calloc((size_t)bu.m * bu.m, sizeof(double));
  bu.hvec = (double *)calloc(bu.m, sizeof(double));
  bu.cvec = (double *)calloc(bu.m, sizeof(double));
  bu.eta = 0.7071; bu.deftol = 10 * ORC_MACHINE_EPS; bu.seed = 0x5eedULL; bu.nrand = 0;
  for (j = 0; j < nconv; j++) csr_mult(m, rowptr, colind, vals, X + (size_t)j * n, bu.V + (size_t)j * m);
  for (j = 0; j < nconv && !st; j++) {
    if ((st = orthogonalize_gs(&bu, j, NULL, &norm, &lindep))) break;
    if (norm == 0.0) { st = ORC_ERR_BREAKDOWN; break; }
    scale_column(&bu, j, 1.0 / norm);
  }
  if (!st) {
    double *r1 = (double *)malloc(sizeof(double) * (size_t)m), *r2 = (double *)malloc(sizeof(double) * (size_t)n);
    for (i = 0; i < nconv; i++) {
      const int p = perm[i];
      const double s = sig[p], *u = bu.V + (size_t)p * m, *v = X + (size_t)p * n;
      if (sigma_out) sigma_out[i] = s;
      if (U_out) memcpy(U_out + (size_t)i * m, u, sizeof(double) * (size_t)m);
      if (V_out) memcpy(V_out + (size_t)i * n, v, sizeof(double) * (size_t)n);
      if (rel_error) {
        double n1, n2;
        csr_mult(m, rowptr, colind, vals, v, r1);
        for (j = 0; j < m; j++) r1[j] -= s * u[j];
        csr_mult(n, rowptr_t, colind_t, vals_t, u, r2);
        for (j = 0; j < n; j++) r2[j] -= s * v[j];
        n1 = nrm2(m, r1);
        n2 = nrm2(n, r2);
        rel_error[i] = hypot(n1, n2) / (s * sqrt(2.0));
      }
    }
    free(r1); free(r2);
  }
  free(bu.V); free(bu.buf); free(bu.hvec); free(bu.cvec);
done:
  free(op.w); free(lam); free(sig); free(perm); free(X);
  return st;
}

/* ======================================================================
 * Building blocks exposed for known-answer tests (BV and DS unit level).
 * ====================================================================== */

/* BVOrthogonalizeColumn (bvorthog.c:315-340) on a caller-owned V (ld x m).
 * H receives j+1 values (coefficients, then the norm), as BV_StoreCoefficients. */
int oracle_bv_orthogonalize_column(int n, int m, int ld, double *V, int j, double *H, double *norm, int *lindep)
{
  obv bv;
  int st, lnd = 0;
  double nrm = 0.0;
  bv.n = n; bv.m = m; bv.ld = ld; bv.V = V;
  bv.buf = (double *)calloc((size_t)m * m, sizeof(double));
  bv.hvec = (double *)calloc(m + 1, sizeof(double));
  bv.cvec = (double *)calloc(m + 1, sizeof(double));
  bv.eta = 0.7071; bv.deftol = 10 * ORC_MACHINE_EPS; bv.seed = 0x5eedULL; bv.nrand = 0;
  st = orthogonalize_gs(&bv, j, NULL, &nrm, &lnd);
  if (!st && H) for (int i = 0; i <= j; i++) H[i] = bv.buf[i + (size_t)j * m];
  if (norm) *norm = nrm;
  if (lindep) *lindep = lnd;
  free(bv.buf); free(bv.hvec); free(bv.cvec);
  return st;
}

/* BVOrthonormalizeColumn (bvorthog.c:380-427): orthogonalize then scale by 1/norm */
int oracle_bv_orthonormalize_column(int n, int m, int ld, double *V, int j, double *H, double *norm, int *lindep)
{
  double nrm = 0.0;
  int st = oracle_bv_orthogonalize_column(n, m, ld, V, j, H, &nrm, lindep);
  if (st) return st;
  if (nrm != 1.0 && nrm != 0.0) {
    double alpha = 1.0 / nrm;
    for (int i = 0; i < n; i++) V[i + (size_t)j * ld] *= alpha;
  }
  if (norm) *norm = nrm;
  return ORC_OK;
}

/* BVOrthogonalizeVec (bvorthog.c:238-262): v against the k active columns of V */
int oracle_bv_orthogonalize_vec(int n, int k, int ld, const double *V, double *v, double *H, double *norm, int *lindep)
{
  obv bv;
  int st, lnd = 0;
  double nrm = 0.0;
  bv.n = n; bv.m = k; bv.ld = ld; bv.V = (double *)V;
  bv.buf = NULL;
  bv.hvec = (double *)calloc(k + 1, sizeof(double));
  bv.cvec = (double *)calloc(k + 1, sizeof(double));
  bv.eta = 0.7071; bv.deftol = 10 * ORC_MACHINE_EPS; bv.seed = 0x5eedULL; bv.nrand = 0;
  st = orthogonalize_gs(&bv, k, v, &nrm, &lnd);
  if (!st && H) for (int i = 0; i < k; i++) H[i] = bv.hvec[i];
  if (norm) *norm = nrm;
  if (lindep) *lindep = lnd;
  free(bv.hvec); free(bv.cvec);
  return st;
}

/* BVMultInPlace_BLAS_Private (bvblas.c:74-106): V(:,s:e) = V(:,l:k) * Q(l:k,s:e) */
int oracle_bv_multinplace(int n, int ld, double *V, int l, int k, const double *Q, int ldq, int s, int e)
{
  int ncols = e - s, kq = k - l, bs = 64, rr, j;
  const double one = 1.0, zero = 0.0;
  if (ncols <= 0 || kq <= 0 || n <= 0) return ORC_OK;
  double *work = (double *)malloc(sizeof(double) * (size_t)bs * ncols);
  const double *pb = Q + (size_t)l + (size_t)s * ldq;
  double *A = V + (size_t)l * ld;
  int r0 = n % bs;
  if (r0) {
    scipy_dgemm_("N", "N", &r0, &ncols, &kq, &one, A, &ld, pb, &ldq, &zero, work, &r0, 1, 1);
    for (j = 0; j < ncols; j++) memcpy(V + (size_t)(s + j) * ld, work + (size_t)j * r0, sizeof(double) * r0);
  }
  for (rr = r0; rr < n; rr += bs) {
    scipy_dgemm_("N", "N", &bs, &ncols, &kq, &one, A + rr, &ld, pb, &ldq, &zero, work, &bs, 1, 1);
    for (j = 0; j < ncols; j++) memcpy(V + (size_t)(s + j) * ld + rr, work + (size_t)j * bs, sizeof(double) * bs);
  }
  free(work);
  return ORC_OK;
}

/* DSSolve_HEP_QR on a dense symmetric A (non-compact path: sytrd + orgtr + steqr,
 * dshep.c:289-307 and :383-427) followed by DSSort_HEP.  Outputs sorted wr and Q. */
int oracle_ds_hep_dense(int n, int ld, const double *A, int which, double *wr, double *Q)
{
  int info = 0, lwork = ld * ld, i;
  double *d = (double *)calloc(ld, sizeof(double)), *e = (double *)calloc(ld, sizeof(double));
  double *tau = (double *)calloc(ld, sizeof(double)), *work = (double *)calloc((size_t)lwork + 64, sizeof(double));
  double *rwork = (double *)calloc(2 * ld + 2, sizeof(double));
  ods ds;
  int st = ORC_OK;
  memset(Q, 0, sizeof(double) * (size_t)ld * ld);
  for (int c = 0; c < n; c++) for (int r = 0; r < n; r++) Q[r + (size_t)c * ld] = A[r + (size_t)c * ld];
  scipy_dsytrd_("L", &n, Q, &ld, d, e, tau, work, &lwork, &info, 1);
  if (info) { st = ORC_ERR_LAPACK; goto out; }
  scipy_dorgtr_("L", &n, Q, &ld, tau, work, &lwork, &info, 1);
  if (info) { st = ORC_ERR_LAPACK; goto out; }
  scipy_dsteqr_("V", &n, d, e, Q, &ld, rwork, &info, 1);
  if (info) { st = ORC_ERR_LAPACK; goto out; }
  ds.ld = ld; ds.n = n; ds.l = 0; ds.k = 0; ds.t = n; ds.which = which; ds.d = d; ds.e = e; ds.Q = Q;
  ds.perm = (int *)calloc(ld, sizeof(int));
  ds_sort_hep(&ds, wr);
  free(ds.perm);
  for (i = 0; i < n; i++) wr[i] = d[i];
out:
  free(d); free(e); free(tau); free(work); free(rwork);
  return st;
}

/* Compact HEP solve of an arrowhead+tridiagonal T (d,e with arrow rows l..k-1),
 * as used inside Krylov-Schur: DSSolve + DSSort + DSUpdateExtraRow. */
int oracle_ds_hep_compact(int ld, int n, int l, int k, int raw, int which, double *d, double *e, double *Q, double *wr)
{
  ods ds;
  int st;
  ds.ld = ld; ds.n = n; ds.l = l; ds.k = k; ds.t = n; ds.state = raw ? 0 : 1; ds.which = which;
  ds.d = d; ds.e = e; ds.Q = Q;
  ds.rwork = (double *)calloc(2 * ld + 2, sizeof(double));
  ds.perm = (int *)calloc(ld, sizeof(int));
  st = ds_solve_hep_qr(&ds, wr);
  if (!st) { ds_sort_hep(&ds, wr); ds_update_extra_row(&ds); }
  free(ds.rwork); free(ds.perm);
  return st;
}

/* Relative residual ||A x - lambda x|| / |lambda| (EPSComputeError, epssolve.c:742-838,
 * EPSComputeResidualNorm_Private :666-722) */
double oracle_residual(int n, const int *rowptr, const int *colind, const double *vals, const double *x, double lambda)
{
  double *u = (double *)malloc(sizeof(double) * (size_t)n), r;
  oracle_spmv(n, rowptr, colind, vals, x, u);
  if (fabs(lambda) > ORC_MACHINE_EPS) for (int i = 0; i < n; i++) u[i] -= lambda * x[i];
  r = nrm2(n, u);
  free(u);
  return r / fabs(lambda);
}

/* ======================================================================
 * LOBPCG: EPSSolve_LOBPCG (src/eps/impls/cg/lobpcg/lobpcg.c:86-398) with
 * EPSSetUp_LOBPCG / EPSSetDimensions_LOBPCG (:40-84), soft and hard locking,
 * a standard symmetric problem (B = NULL), and the preconditioner of
 * STPRECOND + KSPPREONLY: PCNONE (identity) or PCJACOBI (w = diag(A)^{-1} r,
 * zero diagonal entries replaced by 1).  The block operations follow the BV
 * interface with active columns [l,k):
 *   BVCopy (bvbasic.c:1779, BVCopy_Svec svec.c:233-247), BVMatMult
 *   (bvops.c), BVMatProject_MatMult / _Dot (bvglobal.c:902-1060), BVDot and
 *   BVMult (BLAS gemm, bvblas.c), BVMultInPlace (64-row blocked gemm),
 *   BVOrthogonalize_GS (bvorthog.c:507-548: each column against ALL previous
 *   columns, leading ones included), BVOrthogonalizeVec (:238-262),
 *   BVInsertVecs (bvfunc.c:331-374);
 * DSGHEP: LAPACK dsygvd itype 1 "V" "U" (dsghep.c:96-148), DSSort_GHEP
 * (:75-94, insertion sort with SlepcCompareSmallestReal; the spectrum is
 * flipped for the largest), DSVectors_GHEP (X = Q).
 * ====================================================================== */
extern void scipy_dsygvd_(const int *, const char *, const char *, const int *, double *, const int *, double *,
                          const int *, double *, double *, const int *, int *, const int *, int *, size_t, size_t);

typedef struct {
  obv b;     /* storage and Gram-Schmidt scratch */
  int l, k;  /* active columns */
} oblk;

#define BCOL(B, j) ((B)->b.V + (size_t)(j) * (B)->b.ld)

static void blk_init(oblk *B, int n, int m)
{
  B->b.n = n; B->b.m = m; B->b.ld = n;
  B->b.V = (double *)calloc((size_t)n * m, sizeof(double));
  B->b.buf = (double *)calloc((size_t)m * m, sizeof(double));
  B->b.hvec = (double *)calloc((size_t)m + 1, sizeof(double));
  B->b.cvec = (double *)calloc((size_t)m + 1, sizeof(double));
  B->b.eta = 0.7071; B->b.deftol = 10 * ORC_MACHINE_EPS; B->b.seed = 0x5eedULL; B->b.nrand = 0;
  B->l = 0; B->k = m;
}

static void blk_free(oblk *B)
{
  free(B->b.V); free(B->b.buf); free(B->b.hvec); free(B->b.cvec);
}

static void blk_active(oblk *B, int l, int k) { B->l = l; B->k = k; }

static void blk_copy(const oblk *src, oblk *dst)
{
  for (int j = 0; j < src->k - src->l; j++)
    memcpy(BCOL(dst, dst->l + j), BCOL(src, src->l + j), sizeof(double) * (size_t)src->b.n);
}

static void blk_copy_column(oblk *B, int j, int i)
{
  memcpy(BCOL(B, i), BCOL(B, j), sizeof(double) * (size_t)B->b.n);
}

static void blk_matmult(const orc_op *op, const oblk *X, oblk *Y)
{
  for (int j = 0; j < X->k - X->l; j++) op_apply(op, BCOL(X, X->l + j), BCOL(Y, Y->l + j));
}

/* M(Y.l+i, X.l+j) = Y(:,Y.l+i)' X(:,X.l+j) (BVDot: M = Y^H X on active columns) */
static void blk_dot(const oblk *X, const oblk *Y, double *M, int ldm)
{
  const int nx = X->k - X->l, ny = Y->k - Y->l, n = X->b.n;
  const double one = 1.0, zero = 0.0;
  if (nx <= 0 || ny <= 0) return;
  scipy_dgemm_("T", "N", &ny, &nx, &n, &one, BCOL(Y, Y->l), &Y->b.ld, BCOL(X, X->l), &X->b.ld, &zero,
               M + Y->l + (size_t)X->l * ldm, &ldm, 1, 1);
}

/* BVMult: Y(:,Y.l:Y.k) = beta Y + alpha X(:,X.l:X.k) Q(X.l:X.k, Y.l:Y.k) */
static void blk_mult(oblk *Y, double alpha, double beta, const oblk *X, const double *Q, int ldq)
{
  const int nx = X->k - X->l, ny = Y->k - Y->l, n = X->b.n;
  if (ny <= 0) return;
  if (nx <= 0) { for (int j = 0; j < ny; j++) for (int i = 0; i < n; i++) BCOL(Y, Y->l + j)[i] *= beta; return; }
  scipy_dgemm_("N", "N", &n, &ny, &nx, &alpha, BCOL(X, X->l), &X->b.ld, Q + X->l + (size_t)Y->l * ldq, &ldq, &beta,
               BCOL(Y, Y->l), &Y->b.ld, 1, 1);
}

/* BVMultInPlace(V,Q,s,e): V(:,s:e) = V(:,l:k) Q(l:k,s:e), 64-row blocks (bvblas.c:74-106) */
static void blk_multinplace(oblk *V, const double *Q, int ldq, int s, int e)
{
  int ncols = e - s, kq = V->k - V->l, bs = 64, rr, j, n = V->b.n;
  const double one = 1.0, zero = 0.0;
  if (ncols <= 0 || kq <= 0) return;
  double *work = (double *)malloc(sizeof(double) * (size_t)bs * ncols);
  const double *pb = Q + V->l + (size_t)s * ldq;
  double *A = BCOL(V, V->l);
  int r0 = n % bs;
  if (r0) {
    scipy_dgemm_("N", "N", &r0, &ncols, &kq, &one, A, &V->b.ld, pb, &ldq, &zero, work, &r0, 1, 1);
    for (j = 0; j < ncols; j++) memcpy(BCOL(V, s + j), work + (size_t)j * r0, sizeof(double) * r0);
  }
  for (rr = r0; rr < n; rr += bs) {
    scipy_dgemm_("N", "N", &bs, &ncols, &kq, &one, A + rr, &V->b.ld, pb, &ldq, &zero, work, &bs, 1, 1);
    for (j = 0; j < ncols; j++) memcpy(BCOL(V, s + j) + rr, work + (size_t)j * bs, sizeof(double) * bs);
  }
  free(work);
}

/* BVOrthogBlockType (slepcbv.h:84-88) */
#define ORC_BLOCK_GS 0
#define ORC_BLOCK_CHOL 1
#define ORC_BLOCK_SVQB 4

extern void scipy_dpotrf_(const char *, const int *, double *, const int *, int *, size_t);
extern void scipy_dtrtri_(const char *, const char *, const int *, double *, const int *, int *, size_t, size_t);
extern void scipy_dsyev_(const char *, const char *, const int *, double *, const int *, double *, double *,
                         const int *, int *, size_t, size_t);

/* The Gram-matrix block orthogonalizations of the active columns [l,k):
 *   BVOrthogonalize_Chol (bvorthog.c:595-613): BVOrthogonalize_BlockGS against
 *   the leading columns (:492-501, V2 -= V1 (V1' V2), one pass), G = V2' V2,
 *   BVMatCholInv_LAPACK_Private (bvlapack.c:136-213: dpotrf "U", on failure
 *   once more with 50 eps added to the diagonal, then dtrtri "U" "N"),
 *   BVMultInPlace(V, inv(R), l, k);
 *   BVOrthogonalize_SVQB (bvorthog.c:665-684): BlockGS, G = V2' V2,
 *   BVMatSVQB_LAPACK_Private (bvlapack.c:261-340: D = diag(G)^{-1/2}, dsyev
 *   "V" "L" of D G D = U Lambda U', S = D U Lambda^{-1/2}), BVMultInPlace(V, S).
 * R (nullable, ldr >= k): R(0:l, l:k) = V1' V2 and R(l:k, l:k) = the Cholesky
 * factor (upper triangular) or Lambda^{1/2} U' D^{-1} (SVQB), so that
 * V_in = V_out R.  A zero column or a non-positive eigenvalue of the SVQB Gram
 * matrix (a numerically rank-deficient block) is reported as ORC_ERR_BREAKDOWN. */
static int blk_orthogonalize_gram(oblk *B, int type, double *Rout, int ldr)
{
  const int l = B->l, nc = B->k - B->l, n = B->b.n, ld = B->b.ld;
  const double one = 1.0, zero = 0.0, mone = -1.0;
  int info = 0, st = ORC_OK, i, j;
  if (nc <= 0) return ORC_OK;
  double *C = NULL, *G = (double *)malloc(sizeof(double) * (size_t)nc * nc);
  double *S = (double *)calloc((size_t)nc * nc, sizeof(double));
  double *Rf = (double *)calloc((size_t)nc * nc, sizeof(double));
  double *work = NULL, *eig = NULL, *D = NULL;
  if (l > 0) {
    C = (double *)malloc(sizeof(double) * (size_t)l * nc);
    scipy_dgemm_("T", "N", &l, &nc, &n, &one, B->b.V, &ld, BCOL(B, l), &ld, &zero, C, &l, 1, 1);
    scipy_dgemm_("N", "N", &n, &nc, &l, &mone, B->b.V, &ld, C, &l, &one, BCOL(B, l), &ld, 1, 1);
  }
  scipy_dgemm_("T", "N", &nc, &nc, &n, &one, BCOL(B, l), &ld, BCOL(B, l), &ld, &zero, G, &nc, 1, 1);
  if (type == ORC_BLOCK_CHOL) {
    memcpy(Rf, G, sizeof(double) * (size_t)nc * nc);
    scipy_dpotrf_("U", &nc, Rf, &nc, &info, 1);
    if (info) {
      memcpy(Rf, G, sizeof(double) * (size_t)nc * nc);
      for (i = 0; i < nc; i++) Rf[i + (size_t)i * nc] += 50.0 * ORC_MACHINE_EPS;
      info = 0;
      scipy_dpotrf_("U", &nc, Rf, &nc, &info, 1);
      if (info) { st = ORC_ERR_LAPACK; goto out; }
    }
    for (j = 0; j < nc; j++)
      for (i = j + 1; i < nc; i++) Rf[i + (size_t)j * nc] = 0.0;
    memcpy(S, Rf, sizeof(double) * (size_t)nc * nc);
    scipy_dtrtri_("U", "N", &nc, S, &nc, &info, 1, 1);
    if (info) { st = ORC_ERR_LAPACK; goto out; }
  } else {
    int lwork = -1;
    double q;
    eig = (double *)malloc(sizeof(double) * (size_t)nc);
    D = (double *)malloc(sizeof(double) * (size_t)nc);
    scipy_dsyev_("V", "L", &nc, S, &nc, eig, &q, &lwork, &info, 1, 1);
    lwork = (int)q;
    work = (double *)malloc(sizeof(double) * (size_t)(lwork > 1 ? lwork : 1));
    for (i = 0; i < nc; i++) {
      if (!(G[i + (size_t)i * nc] > 0.0)) { st = ORC_ERR_BREAKDOWN; goto out; }
      D[i] = 1.0 / sqrt(G[i + (size_t)i * nc]);
    }
    for (j = 0; j < nc; j++)
      for (i = 0; i < nc; i++) S[i + (size_t)j * nc] = G[i + (size_t)j * nc] * D[i] * D[j];
    scipy_dsyev_("V", "L", &nc, S, &nc, eig, work, &lwork, &info, 1, 1);
    if (info) { st = ORC_ERR_LAPACK; goto out; }
    for (i = 0; i < nc; i++)
      if (!(eig[i] > 0.0)) { st = ORC_ERR_BREAKDOWN; goto out; }
    /* R = Lambda^{1/2} U' / D, S = D U Lambda^{-1/2} */
    for (j = 0; j < nc; j++)
      for (i = 0; i < nc; i++) Rf[i + (size_t)j * nc] = S[j + (size_t)i * nc] * sqrt(eig[i]) / D[j];
    for (j = 0; j < nc; j++)
      for (i = 0; i < nc; i++) S[i + (size_t)j * nc] = S[i + (size_t)j * nc] * D[i] / sqrt(eig[j]);
  }
  {
    /* BVMultInPlace(V, S, l, k): Q indexed from the active columns */
    const int ldq = B->k;
    double *Q = (double *)calloc((size_t)ldq * ldq, sizeof(double));
    for (j = 0; j < nc; j++) memcpy(Q + l + (size_t)(l + j) * ldq, S + (size_t)j * nc, sizeof(double) * (size_t)nc);
    blk_multinplace(B, Q, ldq, l, B->k);
    free(Q);
  }
  if (Rout) {
    for (j = 0; j < nc; j++) {
      for (i = 0; i < l; i++) Rout[i + (size_t)(l + j) * ldr] = C[i + (size_t)j * l];
      for (i = 0; i < nc; i++) Rout[l + i + (size_t)(l + j) * ldr] = Rf[i + (size_t)j * nc];
    }
  }
out:
  free(C); free(G); free(S); free(Rf); free(work); free(eig); free(D);
  return st;
}

/* BVOrthogonalize (bvorthog.c:726-767) with the given BVOrthogBlockType; BV_ORTHOG_BLOCK_GS
 * proceeds column by column (BVOrthogonalize_GS, :507-548). */
static int blk_orthogonalize(oblk *B, int type)
{
  double norm;
  int lindep, st;
  if (type == ORC_BLOCK_CHOL || type == ORC_BLOCK_SVQB) return blk_orthogonalize_gram(B, type, NULL, 0);
  if (type != ORC_BLOCK_GS) return ORC_ERR_ARG;
  for (int j = B->l; j < B->k; j++) {
    if ((st = orthogonalize_gs(&B->b, j, NULL, &norm, &lindep))) return st;
    if (norm == 0.0) return ORC_ERR_BREAKDOWN;
    scale_column(&B->b, j, 1.0 / norm);
  }
  return ORC_OK;
}

/* BVOrthogonalize of the columns [l,k) of V (n x k, leading dimension ld) with
 * block type 1 (Cholesky) or 4 (SVQB); R as above (nullable). */
int oracle_bv_orthogonalize_block(int n, int ld, double *V, int l, int k, int type, double *R, int ldr)
{
  oblk B;
  if (n <= 0 || ld < n || l < 0 || k < l || (type != ORC_BLOCK_CHOL && type != ORC_BLOCK_SVQB)) return ORC_ERR_ARG;
  memset(&B, 0, sizeof(B));
  B.b.n = n; B.b.m = k; B.b.ld = ld; B.b.V = V;
  B.l = l; B.k = k;
  return blk_orthogonalize_gram(&B, type, R, ldr);
}

/* DSSolve_GHEP + DSSort_GHEP + DSVectors_GHEP on an nv x nv pencil (A, B), ld x ld.
 * On return wr holds the sorted eigenvalues and X (ld x ld) the eigenvectors. */
static int ds_ghep(int nv, int ld, double *A, double *B, double *wr, double *X, int *perm)
{
  int itype = 1, info = 0, n1 = nv, lwork = 2 * nv * nv + 6 * nv + 1, liwork = 5 * nv + 3, i, j, p, k;
  double *work = (double *)malloc(sizeof(double) * (size_t)lwork), rtmp;
  int *iwork = (int *)malloc(sizeof(int) * (size_t)liwork);
  scipy_dsygvd_(&itype, "V", "U", &n1, A, &ld, B, &ld, wr, work, &lwork, iwork, &liwork, &info, 1, 1);
  free(work); free(iwork);
  if (info) return ORC_ERR_LAPACK;
  memset(X, 0, sizeof(double) * (size_t)ld * ld);
  for (i = 0; i < nv; i++) memcpy(X + (size_t)i * ld, A + (size_t)i * ld, sizeof(double) * nv);
  /* insertion sort, smallest real first */
  for (i = 0; i < nv; i++) perm[i] = i;
  for (i = 1; i < nv; i++) {
    double re = wr[perm[i]];
    j = i - 1;
    int result = sc_compare(ORC_SMALLEST_REAL, re, wr[perm[j]]);
    while (result < 0 && j >= 0) {
      int tmp = perm[j]; perm[j] = perm[j + 1]; perm[j + 1] = tmp; j--;
      if (j >= 0) result = sc_compare(ORC_SMALLEST_REAL, re, wr[perm[j]]);
    }
  }
  {
    double *w2 = (double *)malloc(sizeof(double) * (size_t)nv);
    for (i = 0; i < nv; i++) w2[i] = wr[perm[i]];
    memcpy(wr, w2, sizeof(double) * (size_t)nv);
    free(w2);
  }
  for (i = 0; i < nv; i++) {
    p = perm[i];
    if (p != i) {
      j = i + 1;
      while (perm[j] != i) j++;
      perm[j] = p; perm[i] = i;
      for (k = 0; k < nv; k++) {
        rtmp = X[k + (size_t)p * ld]; X[k + (size_t)p * ld] = X[k + (size_t)i * ld]; X[k + (size_t)i * ld] = rtmp;
      }
    }
  }
  return ORC_OK;
}

/* W(:,j) = dinv .* R(:,j) on active columns (PCApply_Jacobi: pointwise product with the inverse diagonal) */
static void precond_apply(const double *dinv, oblk *R)
{
  if (!dinv) return;
  for (int j = R->l; j < R->k; j++) {
    double *w = BCOL(R, j);
    for (int i = 0; i < R->b.n; i++) w[i] = dinv[i] * w[i];
  }
}

/*
 * oracle_lobpcg: EPSSolve with EPSLOBPCG on a symmetric CSR matrix.
 *   which: ORC_SMALLEST_REAL or ORC_LARGEST_REAL; bs <= 0: min(16, nev);
 *   ncv <= 0: the LOBPCG default; restart 0.9; lock 1; max_it <= 0: max(100, 2n/ncv);
 *   pc: 0 none, 1 Jacobi; orthog_block: the BVOrthogBlockType of X, R and P (0 GS, 1 Cholesky,
 *   4 SVQB; BVSetOrthogonalization on eps->V, which the blocks inherit through BVDuplicate);
 *   X0 (n x nini, column-major) the initial space (may be NULL).
 * Outputs sorted eigenvalues (nconv), eigenvectors X (n x nconv), error estimates,
 * info[0..3] = nconv, its, reason, iterations of the inner loop.
 */
int oracle_lobpcg(int n, const int *rowptr, const int *colind, const double *vals, int nev, int bs, int ncv,
                  double tol, int max_it, int which, int pc, int lock, double restart, int orthog_block,
                  const double *X0, int nini, double *evals, double *Xout, double *errest_out, int *info)
{
  orc_op op;
  oblk V, Z, X, R, P, AX, Y;
  int st = ORC_OK, i, j, k, nv, ini, nconv, locked, its, guard, flip, useY, mpd, eps_its = 0, eps_nconv = 0;
  int reason = ORC_ITERATING;
  double *eigr, *errest, *dinv = NULL, *MA, *MB, *Q, *wr, norm;
  int *dsperm, *perm;
  memset(&op, 0, sizeof(op));
  op.n = n; op.rp = rowptr; op.ci = colind; op.va = vals;
  if (which != ORC_SMALLEST_REAL && which != ORC_LARGEST_REAL) return ORC_ERR_ARG;
  if (orthog_block != ORC_BLOCK_GS && orthog_block != ORC_BLOCK_CHOL && orthog_block != ORC_BLOCK_SVQB)
    return ORC_ERR_ARG;
  if (bs <= 0) bs = nev < 16 ? nev : 16;
  k = 3 * bs > ((nev - 1) / bs + 3) * bs ? 3 * bs : ((nev - 1) / bs + 3) * bs;
  if (ncv <= 0) ncv = k;
  else if (ncv < k) return ORC_ERR_ARG;
  mpd = 3 * bs;
  if (n < 5 * bs) return ORC_ERR_ARG;
  if (max_it <= 0) max_it = (2 * n / ncv > 100) ? 2 * n / ncv : 100;
  if (tol <= 0.0) tol = 1e-8;
  if (restart <= 0.0) restart = 0.9;
  guard = bs == 1 ? 0 : (int)((1.0 - restart) * bs + 0.45);
  if (guard > bs - 1) guard = bs - 1;
  flip = which == ORC_LARGEST_REAL;
  useY = nev > bs - guard;

  blk_init(&V, n, ncv);
  blk_init(&Z, n, 3 * bs); blk_init(&X, n, bs); blk_init(&R, n, bs); blk_init(&P, n, bs); blk_init(&AX, n, bs);
  blk_init(&Y, n, useY ? nev : 1);
  blk_active(&Y, 0, 0);
  eigr = (double *)calloc((size_t)ncv + 3 * bs, sizeof(double));
  errest = (double *)calloc((size_t)ncv + 3 * bs, sizeof(double));
  perm = (int *)calloc((size_t)ncv, sizeof(int));
  MA = (double *)calloc((size_t)mpd * mpd, sizeof(double));
  MB = (double *)calloc((size_t)mpd * mpd, sizeof(double));
  Q = (double *)calloc((size_t)mpd * mpd, sizeof(double));
  wr = (double *)calloc((size_t)mpd, sizeof(double));
  dsperm = (int *)calloc((size_t)mpd, sizeof(int));
  if (pc == 1) {
    dinv = (double *)malloc(sizeof(double) * (size_t)n);
    for (i = 0; i < n; i++) {
      double d = 0.0;
      for (int p = rowptr[i]; p < rowptr[i + 1]; p++)
        if (colind[p] == i) d += vals[p];
      dinv[i] = 1.0 / (d != 0.0 ? d : 1.0);
    }
  }

  /* EPSSetUp: BVInsertVecs(V,0,&nini,IS,TRUE) */
  {
    int ndep = 0, lindep;
    for (i = 0; i < nini; i++) {
      memcpy(BCOL(&V, i - ndep), X0 + (size_t)i * n, sizeof(double) * (size_t)n);
      if ((st = orthogonalize_gs(&V.b, i - ndep, NULL, &norm, &lindep))) goto done;
      if (norm == 0.0 || lindep) ndep++;
      else scale_column(&V.b, i - ndep, 1.0 / norm);
    }
    nini -= ndep;
  }
  /* 2-3: more initial vectors */
  for (k = nini; k < ncv - bs; k++) {
    set_random_column(&V.b, k);
    if ((st = orthonormalize_column(&V.b, k, NULL, NULL))) goto done;
  }
  nv = bs;
  blk_active(&V, 0, nv); blk_active(&Z, 0, nv);
  blk_copy(&V, &Z);
  blk_copy(&Z, &X);

  /* 4. initial Ritz vectors */
#define LOBPCG_RAYLEIGH_RITZ_X()                                                         \
  do {                                                                                   \
    blk_matmult(&op, &X, &AX);                                                           \
    memset(MA, 0, sizeof(double) * (size_t)mpd * mpd);                                   \
    blk_dot(&AX, &X, MA, mpd);                                                           \
    if (flip) for (i = 0; i < mpd * mpd; i++) MA[i] = -MA[i];                            \
    memset(MB, 0, sizeof(double) * (size_t)mpd * mpd);                                   \
    for (i = 0; i < nv; i++) MB[i + (size_t)i * mpd] = 1.0;                              \
    if ((st = ds_ghep(nv, mpd, MA, MB, wr, Q, dsperm))) goto done;                       \
    for (j = 0; j < nv; j++) if (locked + j < ncv) eigr[locked + j] = flip ? -wr[j] : wr[j]; \
    blk_multinplace(&X, Q, mpd, 0, nv);                                                  \
    blk_multinplace(&AX, Q, mpd, 0, nv);                                                 \
  } while (0)
  locked = 0;
  LOBPCG_RAYLEIGH_RITZ_X();

  /* 5 */
  nconv = 0;
  its = 0;

  /* 6. main loop */
  while (reason == ORC_ITERATING) {
    if (lock) { blk_active(&R, nconv, bs); blk_active(&AX, nconv, bs); }
    /* 7. residuals */
    ini = lock ? nconv : 0;
    blk_copy(&AX, &R);
    for (j = ini; j < bs; j++) {
      double *r = BCOL(&R, j), *x = BCOL(&X, j), lam = eigr[locked + j];
      for (i = 0; i < n; i++) r[i] -= lam * x[i];   /* VecAXPY */
    }
    /* 8. residual norms, active set */
    k = ini;
    {
      int countc = 1;
      for (j = ini; j < bs; j++) {
        i = locked + j;
        norm = nrm2(n, BCOL(&R, j));
        errest[i] = (eigr[i] != 0.0) ? norm / fabs(eigr[i]) : DBL_MAX;   /* EPSConvergedRelative */
        if (countc) {
          if (errest[i] < tol) k++;
          else countc = 0;
        }
        if (!countc) break;
      }
    }
    nconv = k;
    eps_nconv = locked + nconv;
    /* EPSStoppingBasic */
    if (eps_nconv >= nev) reason = ORC_CONVERGED_TOL;
    else if (eps_its + its >= max_it) reason = ORC_DIVERGED_ITS;
    if (reason != ORC_ITERATING || nconv >= bs - guard) {
      blk_active(&V, locked, eps_nconv);
      blk_active(&X, 0, nconv);
      blk_copy(&X, &V);
    }
    if (reason != ORC_ITERATING) break;
    else if (nconv >= bs - guard) { eps_its += its - 1; its = 0; }
    else its++;

    if (nconv >= bs - guard) {  /* hard locking */
      int lindep;
      blk_active(&Y, locked, locked + nconv);
      blk_copy(&X, &Y);
      blk_active(&Y, 0, locked + nconv);
      for (j = nconv; j < bs; j++) {
        blk_copy_column(&X, j, j - nconv);
        blk_copy_column(&R, j, j - nconv);
        blk_copy_column(&P, j, j - nconv);
        blk_copy_column(&AX, j, j - nconv);
      }
      blk_active(&V, locked + bs, locked + bs + nconv);
      blk_active(&X, bs - nconv, bs);
      blk_copy(&V, &X);
      for (j = bs - nconv; j < bs; j++) {
        double *v = BCOL(&X, j);
        if ((st = orthogonalize_gs(&Y.b, Y.k, v, &norm, &lindep))) goto done;
        if (norm > 0.0 && !lindep) for (i = 0; i < n; i++) v[i] *= 1.0 / norm;   /* VecScale */
        else { reason = ORC_DIVERGED_BREAKDOWN; goto diverged; }
      }
      locked += nconv;
      nconv = 0;
      blk_active(&X, nconv, bs);
      if ((st = blk_orthogonalize(&X, orthog_block))) goto done;
      blk_active(&Z, nconv, bs);
      blk_active(&AX, nconv, bs);
      blk_copy(&X, &Z);
      nv = bs;
      LOBPCG_RAYLEIGH_RITZ_X();
      continue;
    }

    ini = lock ? nconv : 0;
    if (lock) { blk_active(&R, nconv, bs); blk_active(&P, nconv, bs); blk_active(&AX, nconv, bs); }

    /* 9. preconditioner */
    precond_apply(dinv, &R);
    if (locked > 0) {
      int lindep;
      for (j = ini; j < bs; j++) {
        double *w = BCOL(&R, j);
        if ((st = orthogonalize_gs(&Y.b, Y.k, w, &norm, &lindep))) goto done;
        if (norm > 0.0 && !lindep) for (i = 0; i < n; i++) w[i] *= 1.0 / norm;
        if (norm <= 0.0 || lindep) { reason = ORC_DIVERGED_BREAKDOWN; goto diverged; }
      }
    }
    /* 11 */
    if ((st = blk_orthogonalize(&R, orthog_block))) goto done;
    /* 13-16 */
    if (its > 1 && (st = blk_orthogonalize(&P, orthog_block))) goto done;
    /* 17-23 */
    blk_active(&Z, 0, bs); blk_active(&X, 0, bs);
    blk_copy(&X, &Z);
    blk_active(&Z, bs, 2 * bs - ini);
    blk_copy(&R, &Z);
    if (its > 1) {
      blk_active(&Z, 2 * bs - ini, 3 * bs - 2 * ini);
      blk_copy(&P, &Z);
    }
    nv = its > 1 ? 3 * bs - 2 * ini : 2 * bs - ini;
    blk_active(&Z, 0, nv);
    {
      oblk W;   /* BVMatProject_MatMult: W = A Z, M = Z' W */
      blk_init(&W, n, nv);
      blk_matmult(&op, &Z, &W);
      memset(MA, 0, sizeof(double) * (size_t)mpd * mpd);
      blk_dot(&W, &Z, MA, mpd);
      blk_free(&W);
    }
    if (flip) for (i = 0; i < mpd * mpd; i++) MA[i] = -MA[i];
    memset(MB, 0, sizeof(double) * (size_t)mpd * mpd);
    blk_dot(&Z, &Z, MB, mpd);   /* BVMatProject_Dot */
    /* 24 */
    if ((st = ds_ghep(nv, mpd, MA, MB, wr, Q, dsperm))) goto done;
    for (j = 0; j < nv; j++) if (locked + j < ncv) eigr[locked + j] = flip ? -wr[j] : wr[j];
    /* 25-33 */
    blk_active(&Z, bs, nv);
    if (lock) blk_active(&P, 0, bs);
    blk_mult(&P, 1.0, 0.0, &Z, Q, mpd);
    blk_active(&X, 0, bs);
    blk_copy(&P, &X);
    if (lock) blk_active(&P, nconv, bs);
    blk_active(&Z, 0, bs);
    blk_mult(&X, 1.0, 1.0, &Z, Q, mpd);
    if (lock) blk_active(&X, nconv, bs);
    blk_matmult(&op, &X, &AX);
  }

diverged:
  eps_its += its;
  /* EPSSolve post-processing: SlepcSortEigenvalues */
  for (i = 0; i < eps_nconv; i++) perm[i] = i;
  for (i = eps_nconv - 1; i >= 0; i--) {
    double re = eigr[perm[i]];
    j = i + 1;
    while (j < eps_nconv) {
      if (sc_compare(which, re, eigr[perm[j]]) <= 0) break;
      int tmp = perm[j - 1]; perm[j - 1] = perm[j]; perm[j] = tmp;
      j++;
    }
  }
  for (i = 0; i < eps_nconv; i++) {
    if (evals) evals[i] = eigr[perm[i]];
    if (errest_out) errest_out[i] = errest[perm[i]];
    if (Xout) memcpy(Xout + (size_t)i * n, BCOL(&V, perm[i]), sizeof(double) * (size_t)n);
  }
done:
#undef LOBPCG_RAYLEIGH_RITZ_X
  if (info) { info[0] = eps_nconv; info[1] = eps_its; info[2] = reason; info[3] = ncv; }
  blk_free(&V); blk_free(&Z); blk_free(&X); blk_free(&R); blk_free(&P); blk_free(&AX); blk_free(&Y);
  free(eigr); free(errest); free(perm); free(MA); free(MB); free(Q); free(wr); free(dsperm); free(dinv);
  return st;
}

/*
 * oracle_eps_solve_batch: oracle_eps_solve on every problem of a batch, the
 * problems spread over the host threads (each problem single-threaded).
 * rowptr: the problems' local row pointers one after another (ns[p]+1 each);
 * colind/vals: their nonzeros one after another; v0: start vectors one after
 * another.  Outputs per problem p: evals[p*ncv ...] (nconv sorted values),
 * info[p*6 ...] as oracle_eps_solve.  Returns the number of failed problems.
 */
int oracle_eps_solve_batch(int nprob, const int *ns, const int *rowptr, const int *colind, const double *vals,
                           const double *v0, int nev, int ncv, double tol, int which, double *evals, int *info)
{
  long long *rp_off = (long long *)malloc(sizeof(long long) * (size_t)(nprob + 1));
  long long *nz_off = (long long *)malloc(sizeof(long long) * (size_t)(nprob + 1));
  long long *x_off = (long long *)malloc(sizeof(long long) * (size_t)(nprob + 1));
  int p, bad = 0;
  rp_off[0] = nz_off[0] = x_off[0] = 0;
  for (p = 0; p < nprob; p++) {
    rp_off[p + 1] = rp_off[p] + ns[p] + 1;
    nz_off[p + 1] = nz_off[p] + rowptr[rp_off[p] + ns[p]];
    x_off[p + 1] = x_off[p] + ns[p];
  }
#ifdef _OPENMP
  int levels = omp_get_max_active_levels();
  omp_set_max_active_levels(1);
#endif
  scipy_openblas_set_num_threads(1);
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : bad)
  for (p = 0; p < nprob; p++) {
    int st = oracle_eps_solve(ns[p], rowptr + rp_off[p], colind + nz_off[p], vals + nz_off[p], v0 + x_off[p], nev, ncv,
                              0, tol, 0, which, 0, evals + (size_t)p * ncv, NULL, NULL, info + (size_t)p * 6);
    if (st) bad++;
  }
#ifdef _OPENMP
  omp_set_max_active_levels(levels);
#endif
  free(rp_off); free(nz_off); free(x_off);
  return bad;
}
