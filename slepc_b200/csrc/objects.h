// Host objects shared by the C ABI translation units: the Mat (CSR operands
// and the cross shell), the BV (basis in HBM with its Gram-Schmidt work
// arrays) and the EPS solver state (Krylov-Schur or LOBPCG).
#pragma once
#include <cuda_runtime.h>

#include <cstdio>
#include <utility>
#include <vector>

#include "common.h"
#include "ds_hep.h"
#include "kernels.h"

// One CSR operand in HBM with its SpMV schedules.  Values are FP64, or FP32
// (B200_SCALAR_F32: half the value traffic; products and sums stay FP64).
struct CsrPart {
  int rows = 0, cols = 0;
  int64_t nnz = 0;
  int *rowptr = nullptr, *colind = nullptr;
  void *vals = nullptr;
  bool f32 = false;
  int lanes = 8;
  int *blocks = nullptr;       // row blocks of the row-block SpMV (nblocks + 1 entries), FP64 only
  int nblocks = 0;
  b200::SpmvTiles wt;                // warp tiles, long-row segments and their partial-sum slots
  b200::SpmvSell sell;               // sliced-ELL copy (built when that schedule is selected)
  bool sell_ready = false;
  float *vals32 = nullptr;           // FP32 copy of FP64 values for the mixed-precision solver
};

enum MatKind { kMatCsr = 0, kMatCross = 1 };

// kMatCsr: the matrix A (m x n) with, for a rectangular AIJ matrix, its explicit
// transpose.  kMatCross: the shell C = A^T A (n x n) of MatMult_Cross
// (src/svd/impls/cross/cross.c:31-41) over a kMatCsr matrix it does not own.
struct b200_mat_s {
  int kind = kMatCsr;
  int m = 0, n = 0;          // rows and columns of the operator
  int64_t nnz = 0;
  CsrPart a;                 // A
  CsrPart at;                // A^T (rectangular AIJ matrices; rows == 0 otherwise)
  b200_mat base = nullptr;   // kMatCross: the matrix A of A^T A
  bool swapped = false;      // kMatCross: the operator is A A^T (SVDSetUp's swap for m < n)
  double *work = nullptr;    // kMatCross: w = A x (base->m entries; base->n when swapped)
  double norm_inf = -1.0;    // max_i sum_j |a_ij| when known (computed from the host arrays)
  int schedule = B200_SPMV_SELL;
  cudaStream_t stream = nullptr;
};

struct b200_bv_s {
  int n = 0, m = 0, ld = 0;   // m user columns; column m is an internal work column
  double *V = nullptr;
  int l = 0, k = 0;
  double eta = 0.7071;        // bvfunc.c:178
  int orthog_block = B200_ORTHOG_BLOCK_GS;  // bvfunc.c:179
  cudaStream_t stream = nullptr;
  b200::GsWork gs{};
  double *coefbuf = nullptr;  // (m+1) x (m+1): column j = coefficients of column j (BVGetBufferVec)
  int ldc = 0;
  double *hvec = nullptr;     // coefficients of the vector variant
  double *T = nullptr;        // Lanczos alpha (T[j]) and beta (T[ldt+j])
  int ldt = 0;
  double *red = nullptr;      // reduction workspace
  int red_len = 0;
  double *scal = nullptr;     // device scalars
  double *qbuf = nullptr;     // device staging of coefficient matrices
  size_t qbuf_len = 0;
  double *hpin = nullptr;     // pinned host staging
  cudaEvent_t hpin_ev = nullptr;  // recorded after each host-to-device copy out of hpin
  size_t hpin_len = 0;
  uint64_t seed = 0x5eedULL, nrand = 0;
};

static inline double *col(b200_bv bv, int j) { return bv->V + (size_t)j * bv->ld; }

struct b200_eps_s {
  cudaStream_t stream = nullptr;
  b200_mat A = nullptr;
  int nev = 1, ncv = 0, mpd = 0;
  double tol = 0.0;
  int max_it = 0;
  int which = B200_LARGEST_MAGNITUDE;
  double keep = 0.5;  // krylovschur.c:122
  int lock = 1;       // EPSKrylovSchurSetLocking (krylovschur.c:427-434; locking by default)
  std::vector<double> v0;
  const double *v0_dev = nullptr;
  int nini = 0;
  int max_restarts = 0;
  b200_bv V = nullptr;
  b200::DsHep ds;
  std::vector<double> eigr, errest;
  std::vector<int> perm;
  int nconv = 0, its = 0, reason = 0;
  bool solved = false;
  int timing = 0;
  b200_eps_stats stats{};
  // effective values after setup
  int n_ = 0, ncv_ = 0, mpd_ = 0, max_it_ = 0;
  double tol_ = 1e-8;
  double *resid_buf = nullptr;
  double *op_buf = nullptr;  // Op x for residuals of operators without a fused residual kernel
  // solver type and LOBPCG parameters (EPSSetType, EPSLOBPCGSet*, STPRECOND's PC)
  int type = B200_EPS_KRYLOVSCHUR;
  bool which_set = false;
  int lobpcg_bs = 0;
  double lobpcg_restart = 0.0;
  int lobpcg_lock = 1;
  int pc = B200_PC_JACOBI;
  int orthog_block = B200_ORTHOG_BLOCK_GS;  // BVSetOrthogonalization block type of eps->V (LOBPCG blocks)
  std::vector<double> X0;  // initial space of EPSSetInitialSpace with several vectors (n x nini_block)
  int nini_block = 0;
  int nini_eff = 0;  // initial vectors kept by BVInsertVecs in the last setup
  double *dinv = nullptr;  // device inverse diagonal for the Jacobi preconditioner
  const void *dinv_of = nullptr;
  // EPSMonitorSet: host callbacks per outer iteration; the built-in JSON-lines monitor
  std::vector<std::pair<b200_eps_monitor_fn, void *>> monitors;
  FILE *monitor_jsonl = nullptr;
  double monitor_t0 = 0.0;  // host time (ms) at the start of the solve
  // mixed-precision form (b200_eps_set_precision): parameters and device buffers
  int precision = B200_PRECISION_FP64;
  double mixed_tol_low = 0.0;  // tolerance of the FP32 phase (0: default)
  int mixed_degree = 0;        // largest Chebyshev degree of one sweep (0: default)
  int mixed_guard = -1;        // block columns beyond nev (-1: default)
  int mixed_max_sweeps = 0;    // sweeps per phase (0: default)
  int mixed_fp64_gram = 0;     // 1: FP64 Gram for the FP32 phase's orthonormalisation (0: tensor cores)
  float *rb32 = nullptr;       // FP32 row-major blocks (4 x n x block width)
  size_t rb32_cap = 0;
  double *rb64 = nullptr;      // FP64 row-major blocks (4 x n x block width)
  size_t rb64_cap = 0;
  double *mred = nullptr;      // small device matrices and reduction work of the mixed form
  size_t mred_cap = 0;
};

