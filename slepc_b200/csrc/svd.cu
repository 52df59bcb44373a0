// SVD cross solver: SVDSolve with SVDCROSS for a standard (non-generalized,
// non-hyperbolic) problem.
//
// Restates SVDSetUp_Cross (src/svd/impls/cross/cross.c:160-250: EPS_HEP on
// the shell C = A^T A of MatMult_Cross, largest/smallest magnitude, EPS tol =
// SLEPC_DEFAULT_TOL/10 when unset), SVDSolve_Cross (cross.c:256-285: sigma =
// sqrt(lambda) with the negative-eigenvalue check), SVDSolve's sort of the
// singular values (src/svd/interface/svdsolve.c), SVDComputeVectors_Cross and
// SVDComputeVectors_Left (cross.c:346-352, svdsolve.c:21-75: V = the
// eigenvectors, U = A V, BVOrthogonalize(U)), SVDGetSingularTriplet (the u/v
// exchange for m < n) and SVDComputeError with
// SVDComputeResidualNorms_Standard (svdsolve.c:349-369, 485-580).
//
// The eigensolve is the b200_eps Krylov-Schur solver; its operator applies
// the FP32- or FP64-valued A and its explicit transpose with the warp-tile
// SpMV (long rows of the power-law transpose split into segments).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <numeric>
#include <vector>

#include "common.h"
#include "internal.h"
#include "kernels.h"

using namespace b200;

struct b200_svd_s {
  cudaStream_t stream = nullptr;
  b200_mat A = nullptr;    // the matrix of SVDSetOperators (not owned)
  b200_mat C = nullptr;    // cross shell A^T A (or A A^T), owned
  b200_eps eps = nullptr;  // inner Krylov-Schur solver, owned
  b200_bv U = nullptr;     // left vectors of the internal problem: A V orthogonalised, owned
  int nsv = 1, ncv = 0, mpd = 0, max_it = 0;
  double tol = 0.0;
  int which = B200_SVD_LARGEST;
  int timing = 0;
  std::vector<double> v0;
  // solution
  bool solved = false, vectors = false, swapped = false;
  int m = 0, n = 0;  // rows and columns of A
  int nconv = 0, its = 0, reason = 0;
  std::vector<double> sigma;
  std::vector<int> perm;
  double *wl = nullptr, *wr = nullptr;  // residual work vectors (m and n entries)
  int wl_len = 0, wr_len = 0;
  double *red = nullptr;                // reduction partials + two results
};

static constexpr int kSvdRedLen = 1024;
static constexpr double kSqrt2 = 1.4142135623730950488;

extern "C" b200_status b200_svd_create(void *stream, b200_svd *svd) {
  B200_ARG_CHECK(svd, "null argument");
  b200_svd S = new b200_svd_s;
  S->stream = (cudaStream_t)stream;
  *svd = S;
  return B200_OK;
}

extern "C" b200_status b200_svd_destroy(b200_svd svd) {
  if (!svd) return B200_OK;
  b200_bv_destroy(svd->U);
  b200_eps_destroy(svd->eps);
  b200_mat_destroy(svd->C);
  cudaFree(svd->wl);
  cudaFree(svd->wr);
  cudaFree(svd->red);
  delete svd;
  return B200_OK;
}

extern "C" b200_status b200_svd_set_operator(b200_svd svd, b200_mat A) {
  B200_ARG_CHECK(svd && A, "null argument");
  int m = 0, n = 0;
  B200_CHECK(b200_mat_get_sizes(A, &m, &n));
  svd->A = A;
  svd->m = m;
  svd->n = n;
  svd->solved = svd->vectors = false;
  return B200_OK;
}

extern "C" b200_status b200_svd_set_dimensions(b200_svd svd, int nsv, int ncv, int mpd) {
  B200_ARG_CHECK(svd && nsv > 0, "nsv must be positive");
  svd->nsv = nsv;
  svd->ncv = ncv;
  svd->mpd = mpd;
  svd->solved = svd->vectors = false;
  return B200_OK;
}

extern "C" b200_status b200_svd_set_tolerances(b200_svd svd, double tol, int max_it) {
  B200_ARG_CHECK(svd, "null argument");
  svd->tol = tol;
  svd->max_it = max_it;
  svd->solved = svd->vectors = false;
  return B200_OK;
}

extern "C" b200_status b200_svd_set_which_singular_triplets(b200_svd svd, int which) {
  B200_ARG_CHECK(svd && (which == B200_SVD_LARGEST || which == B200_SVD_SMALLEST), "unknown SVDWhich");
  svd->which = which;
  svd->solved = svd->vectors = false;
  return B200_OK;
}

extern "C" b200_status b200_svd_set_initial_space(b200_svd svd, const double *v0) {
  B200_ARG_CHECK(svd && svd->A && v0, "set the operator before the initial space");
  const int dim = svd->m < svd->n ? svd->m : svd->n;
  svd->v0.assign(v0, v0 + dim);
  return B200_OK;
}

extern "C" b200_status b200_svd_set_timing(b200_svd svd, int on) {
  B200_ARG_CHECK(svd, "null argument");
  svd->timing = on;
  return B200_OK;
}

extern "C" b200_status b200_svd_solve(b200_svd svd) {
  B200_ARG_CHECK(svd && svd->A, "SVDSetOperators has not been called");
  svd->solved = svd->vectors = false;
  svd->nconv = svd->its = svd->reason = 0;
  svd->swapped = svd->m < svd->n;
  // SVDSetUp_Cross: the product shell and the inner EPS
  b200_mat_destroy(svd->C);
  svd->C = nullptr;
  B200_CHECK(mat_create_cross_ex(svd->A, svd->swapped, &svd->C));
  if (!svd->eps) B200_CHECK(b200_eps_create(svd->stream, &svd->eps));
  b200_eps E = svd->eps;
  B200_CHECK(b200_eps_set_operators(E, svd->C));
  B200_CHECK(b200_eps_set_which_eigenpairs(
      E, svd->which == B200_SVD_LARGEST ? B200_LARGEST_MAGNITUDE : B200_SMALLEST_MAGNITUDE));
  B200_CHECK(b200_eps_set_dimensions(E, svd->nsv, svd->ncv, svd->mpd));
  B200_CHECK(b200_eps_set_tolerances(E, svd->tol > 0.0 ? svd->tol : 1e-9, svd->max_it));
  if (!svd->v0.empty()) B200_CHECK(b200_eps_set_initial_space(E, svd->v0.data()));
  B200_CHECK(b200_eps_set_timing(E, svd->timing));
  // SVDSolve_Cross
  B200_CHECK(b200_eps_solve(E));
  B200_CHECK(b200_eps_get_converged(E, &svd->nconv));
  B200_CHECK(b200_eps_get_iteration_number(E, &svd->its));
  B200_CHECK(b200_eps_get_converged_reason(E, &svd->reason));
  svd->sigma.assign(svd->nconv, 0.0);
  for (int i = 0; i < svd->nconv; ++i) {
    double lam = 0.0;
    B200_CHECK(b200_eps_get_eigenpair(E, i, &lam, nullptr));
    if (!(lam > -10 * 2.220446049250313e-16)) {
      b200_set_last_error(__FILE__, __LINE__, "negative eigenvalue computed by EPS");
      return B200_ERR_FP;
    }
    svd->sigma[i] = std::sqrt(lam < 0.0 ? 0.0 : lam);
  }
  // SVDSolve: ascending sort, reversed for the largest triplets
  svd->perm.resize(svd->nconv);
  std::iota(svd->perm.begin(), svd->perm.end(), 0);
  std::stable_sort(svd->perm.begin(), svd->perm.end(),
                   [&](int a, int b) { return svd->sigma[a] < svd->sigma[b]; });
  if (svd->which == B200_SVD_LARGEST) std::reverse(svd->perm.begin(), svd->perm.end());
  svd->solved = true;
  return B200_OK;
}

// SVDComputeVectors_Cross + SVDComputeVectors_Left: U = A V, then Gram-Schmidt.
static b200_status svd_compute_vectors(b200_svd svd) {
  if (svd->vectors) return B200_OK;
  const int ulen = svd->swapped ? svd->n : svd->m;  // rows of the internal A
  const int cols = svd->nconv > 0 ? svd->nconv : 1;
  if (svd->U) {
    int bn = 0, bm = 0, ld = 0;
    B200_CHECK(b200_bv_get_sizes(svd->U, &bn, &bm, &ld));
    if (bn != ulen || bm < cols) {
      b200_bv_destroy(svd->U);
      svd->U = nullptr;
    }
  }
  if (!svd->U) B200_CHECK(b200_bv_create(ulen, cols, svd->stream, &svd->U));
  double *Ud = nullptr;
  int ld = 0;
  B200_CHECK(b200_bv_get_array(svd->U, &Ud));
  B200_CHECK(b200_bv_get_sizes(svd->U, nullptr, nullptr, &ld));
  for (int i = 0; i < svd->nconv; ++i) {
    const double *x = nullptr;
    B200_CHECK(b200_eps_get_eigenvector_device(svd->eps, i, &x));
    // internal A = OP (or OP^T when swapped)
    B200_CUDA_CHECK(mat_apply(svd->A, x, Ud + (size_t)i * ld, svd->stream, svd->swapped));
  }
  if (svd->nconv > 0) {
    B200_CHECK(b200_bv_set_active_columns(svd->U, 0, svd->nconv));
    B200_CHECK(b200_bv_orthogonalize(svd->U, nullptr, 0));
  }
  svd->vectors = true;
  return B200_OK;
}

static b200_status svd_check_index(b200_svd svd, int i) {
  if (!svd->solved) {
    b200_set_last_error(__FILE__, __LINE__, "SVDSolve has not been called");
    return B200_ERR_STATE;
  }
  B200_ARG_CHECK(i >= 0 && i < svd->nconv, "index out of range (see b200_svd_get_converged)");
  return B200_OK;
}

extern "C" b200_status b200_svd_get_converged(b200_svd svd, int *nconv) {
  B200_ARG_CHECK(svd && nconv, "null argument");
  *nconv = svd->solved ? svd->nconv : 0;
  return B200_OK;
}

extern "C" b200_status b200_svd_get_iteration_number(b200_svd svd, int *its) {
  B200_ARG_CHECK(svd && its, "null argument");
  *its = svd->its;
  return B200_OK;
}

extern "C" b200_status b200_svd_get_converged_reason(b200_svd svd, int *reason) {
  B200_ARG_CHECK(svd && reason, "null argument");
  *reason = svd->reason;
  return B200_OK;
}

extern "C" b200_status b200_svd_get_singular_vectors_device(b200_svd svd, int i, const double **u, const double **v) {
  B200_ARG_CHECK(svd, "null argument");
  B200_CHECK(svd_check_index(svd, i));
  B200_CHECK(svd_compute_vectors(svd));
  const int p = svd->perm[i];
  double *Ud = nullptr;
  int ld = 0;
  B200_CHECK(b200_bv_get_array(svd->U, &Ud));
  B200_CHECK(b200_bv_get_sizes(svd->U, nullptr, nullptr, &ld));
  const double *left = Ud + (size_t)p * ld;
  const double *right = nullptr;
  B200_CHECK(b200_eps_get_eigenvector_device(svd->eps, p, &right));
  // SVDGetSingularTriplet exchanges u and v when A has fewer rows than columns
  if (u) *u = svd->swapped ? right : left;
  if (v) *v = svd->swapped ? left : right;
  return B200_OK;
}

extern "C" b200_status b200_svd_get_singular_triplet(b200_svd svd, int i, double *sigma, double *u_host,
                                                     double *v_host) {
  B200_ARG_CHECK(svd, "null argument");
  B200_CHECK(svd_check_index(svd, i));
  if (sigma) *sigma = svd->sigma[svd->perm[i]];
  if (!u_host && !v_host) return B200_OK;
  const double *u = nullptr, *v = nullptr;
  B200_CHECK(b200_svd_get_singular_vectors_device(svd, i, &u, &v));
  if (u_host)
    B200_CUDA_CHECK(cudaMemcpyAsync(u_host, u, sizeof(double) * svd->m, cudaMemcpyDeviceToHost, svd->stream));
  if (v_host)
    B200_CUDA_CHECK(cudaMemcpyAsync(v_host, v, sizeof(double) * svd->n, cudaMemcpyDeviceToHost, svd->stream));
  B200_CUDA_CHECK(cudaStreamSynchronize(svd->stream));
  return B200_OK;
}

extern "C" b200_status b200_svd_compute_error(b200_svd svd, int i, int type, double *error) {
  B200_ARG_CHECK(svd && error, "null argument");
  B200_ARG_CHECK(type == B200_ERROR_ABSOLUTE || type == B200_ERROR_RELATIVE || type == B200_ERROR_NORM,
                 "unknown error type");
  B200_CHECK(svd_check_index(svd, i));
  const double s = svd->sigma[svd->perm[i]];
  const double *u = nullptr, *v = nullptr;
  B200_CHECK(b200_svd_get_singular_vectors_device(svd, i, &u, &v));
  if (svd->wl_len < svd->m) {
    cudaFree(svd->wl);
    svd->wl = nullptr;
    B200_CUDA_CHECK(cudaMalloc(&svd->wl, sizeof(double) * (size_t)svd->m));
    svd->wl_len = svd->m;
  }
  if (svd->wr_len < svd->n) {
    cudaFree(svd->wr);
    svd->wr = nullptr;
    B200_CUDA_CHECK(cudaMalloc(&svd->wr, sizeof(double) * (size_t)svd->n));
    svd->wr_len = svd->n;
  }
  if (!svd->red) B200_CUDA_CHECK(cudaMalloc(&svd->red, sizeof(double) * (kSvdRedLen + 2)));
  double *res = svd->red + kSvdRedLen;
  // norm1 = ||A v - sigma u||, norm2 = ||A^T u - sigma v||
  B200_CUDA_CHECK(mat_apply(svd->A, v, svd->wl, svd->stream, false));
  B200_CUDA_CHECK(diff_sumsq_launch(svd->wl, u, s, svd->m, res, svd->red, kSvdRedLen, svd->stream));
  B200_CUDA_CHECK(mat_apply(svd->A, u, svd->wr, svd->stream, true));
  B200_CUDA_CHECK(diff_sumsq_launch(svd->wr, v, s, svd->n, res + 1, svd->red, kSvdRedLen, svd->stream));
  double h[2];
  B200_CUDA_CHECK(cudaMemcpyAsync(h, res, sizeof(h), cudaMemcpyDeviceToHost, svd->stream));
  B200_CUDA_CHECK(cudaStreamSynchronize(svd->stream));
  double err = std::hypot(std::sqrt(h[0]), std::sqrt(h[1]));
  if (type == B200_ERROR_RELATIVE) {
    err /= s * kSqrt2;
  } else if (type == B200_ERROR_NORM) {
    double nrm = 0.0;
    B200_CHECK(b200_mat_norm_inf(svd->A, &nrm));
    err /= nrm * kSqrt2;
  }
  *error = err;
  return B200_OK;
}

extern "C" b200_status b200_svd_get_stats(b200_svd svd, b200_eps_stats *stats) {
  B200_ARG_CHECK(svd && stats && svd->eps, "null argument or no solve yet");
  return b200_eps_get_stats(svd->eps, stats);
}

extern "C" b200_status b200_svd_solve_aij_host(int m, int n, int64_t nnz, const int *rowptr, const int *colind,
                                               const void *vals, int scalar_type, const double *v0, int nsv, int ncv,
                                               double tol, int max_it, double *sigma, double *U, double *V,
                                               double *rel_error, int *info, void *stream) {
  b200_mat A = nullptr;
  b200_svd S = nullptr;
  B200_CHECK(b200_mat_create_aij(m, n, nnz, rowptr, colind, vals, scalar_type, stream, &A));
  b200_status st = b200_svd_create(stream, &S);
  if (st == B200_OK) st = b200_svd_set_operator(S, A);
  if (st == B200_OK) st = b200_svd_set_dimensions(S, nsv, ncv, 0);
  if (st == B200_OK) st = b200_svd_set_tolerances(S, tol, max_it);
  if (st == B200_OK && v0) st = b200_svd_set_initial_space(S, v0);
  if (st == B200_OK) st = b200_svd_solve(S);
  if (st == B200_OK) {
    for (int i = 0; i < S->nconv && st == B200_OK; ++i) {
      st = b200_svd_get_singular_triplet(S, i, sigma ? sigma + i : nullptr, U ? U + (size_t)i * m : nullptr,
                                         V ? V + (size_t)i * n : nullptr);
      if (st == B200_OK && rel_error) st = b200_svd_compute_error(S, i, B200_ERROR_RELATIVE, rel_error + i);
    }
    if (info) {
      b200_eps_stats es{};
      b200_eps_get_stats(S->eps, &es);
      info[0] = S->nconv;
      info[1] = S->its;
      info[2] = S->reason;
      info[3] = (int)es.lanczos_steps;
      info[4] = (int)es.restarts;
    }
  }
  b200_svd_destroy(S);
  b200_mat_destroy(A);
  return st;
}
