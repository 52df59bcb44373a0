// LOBPCG: EPSSolve with EPSLOBPCG for a standard symmetric problem.
//
// Restates EPSSolve_LOBPCG (src/eps/impls/cg/lobpcg/lobpcg.c:86-398) with
// EPSSetUp_LOBPCG / EPSSetDimensions_LOBPCG (:40-84): block size bs
// (default min(16, nev)), ncv = max(3 bs, ((nev-1)/bs + 3) bs), mpd = 3 bs,
// restart 0.9 giving guard vectors, soft locking on, hard locking of a
// block once bs-guard pairs have converged, and the spectrum flipped for the
// largest eigenvalues.  Every block operation has the BV semantics the
// reference relies on (active columns [l,k); BVCopy into the destination's
// leading offset; BVOrthogonalize column by column against ALL previous
// columns, leading ones included; BVMatProject as A Z then Z^T (A Z)).
// The projected pencil is DSGHEP on the host: LAPACK dsygvd, insertion
// sort with the smallest-real comparator, X = Q (dsghep.c:39-148).  The
// preconditioner is STPRECOND + KSPPREONLY with PCNONE or PCJACOBI.
// Vectors stay in HBM; the host holds only the projected matrices.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

#include "common.h"
#include "internal.h"
#include "kernels.h"
#include "objects.h"

extern "C" void scipy_dsygvd_(const int *, const char *, const char *, const int *, double *, const int *, double *,
                              const int *, double *, double *, const int *, int *, const int *, int *, size_t,
                              size_t);

using namespace b200;

namespace {

void active(b200_bv bv, int l, int k) {
  bv->l = l;
  bv->k = k;
}

// BVCopy: W(:, W.l + j) = V(:, V.l + j), j < V.k - V.l
cudaError_t bv_copy(b200_bv V, b200_bv W) {
  const int nc = V->k - V->l;
  if (nc <= 0) return cudaSuccess;
  return cudaMemcpy2DAsync(col(W, W->l), sizeof(double) * W->ld, col(V, V->l), sizeof(double) * V->ld,
                           sizeof(double) * V->n, nc, cudaMemcpyDeviceToDevice, W->stream);
}

cudaError_t bv_copy_column(b200_bv bv, int j, int i) {
  return cudaMemcpyAsync(col(bv, i), col(bv, j), sizeof(double) * bv->n, cudaMemcpyDeviceToDevice, bv->stream);
}

// DSSolve_GHEP + DSSort_GHEP + DSVectors_GHEP on the nv x nv pencil (A, B) with leading
// dimension ld; wr gets the sorted eigenvalues and X (ld x ld) the eigenvectors.
b200_status ds_ghep(int nv, int ld, std::vector<double> &A, std::vector<double> &B, std::vector<double> &wr,
                    std::vector<double> &X) {
  int itype = 1, info = 0, n1 = nv, lwork = 2 * nv * nv + 6 * nv + 1, liwork = 5 * nv + 3;
  std::vector<double> work((size_t)lwork);
  std::vector<int> iwork((size_t)liwork);
  scipy_dsygvd_(&itype, "V", "U", &n1, A.data(), &ld, B.data(), &ld, wr.data(), work.data(), &lwork, iwork.data(),
                &liwork, &info, 1, 1);
  if (info) {
    b200_set_last_error(__FILE__, __LINE__, "LAPACK dsygvd failed");
    return B200_ERR_LAPACK;
  }
  std::fill(X.begin(), X.end(), 0.0);
  for (int i = 0; i < nv; ++i) memcpy(X.data() + (size_t)i * ld, A.data() + (size_t)i * ld, sizeof(double) * nv);
  // insertion sort, smallest real first (DSSortEigenvalues_Private), then DSPermuteColumns_Private
  std::vector<int> perm(nv);
  for (int i = 0; i < nv; ++i) perm[i] = i;
  auto cmp = [](double a, double b) { return (a > b) ? 1 : (a < b) ? -1 : 0; };
  for (int i = 1; i < nv; ++i) {
    const double re = wr[perm[i]];
    int j = i - 1;
    int result = cmp(re, wr[perm[j]]);
    while (result < 0 && j >= 0) {
      std::swap(perm[j], perm[j + 1]);
      --j;
      if (j >= 0) result = cmp(re, wr[perm[j]]);
    }
  }
  std::vector<double> w2(nv);
  for (int i = 0; i < nv; ++i) w2[i] = wr[perm[i]];
  for (int i = 0; i < nv; ++i) wr[i] = w2[i];
  for (int i = 0; i < nv; ++i) {
    const int p = perm[i];
    if (p != i) {
      int j = i + 1;
      while (perm[j] != i) ++j;
      perm[j] = p;
      perm[i] = i;
      for (int k = 0; k < nv; ++k) std::swap(X[k + (size_t)p * ld], X[k + (size_t)i * ld]);
    }
  }
  return B200_OK;
}

struct Blocks {
  b200_bv Z = nullptr, X = nullptr, R = nullptr, P = nullptr, AX = nullptr, Y = nullptr, W = nullptr;
  ~Blocks() {
    b200_bv_destroy(Z);
    b200_bv_destroy(X);
    b200_bv_destroy(R);
    b200_bv_destroy(P);
    b200_bv_destroy(AX);
    b200_bv_destroy(Y);
    b200_bv_destroy(W);
  }
};

}  // namespace

b200_status b200::lobpcg_solve(b200_eps eps) {
  B200_ARG_CHECK(eps->A, "EPSSetOperators must be called first");
  b200_mat A = eps->A;
  const int n = A->n;
  if (!eps->which_set) eps->which = B200_SMALLEST_REAL;
  B200_ARG_CHECK(eps->which == B200_SMALLEST_REAL || eps->which == B200_LARGEST_REAL,
                 "LOBPCG supports only smallest real or largest real eigenvalues");
  const int nev = eps->nev;
  const int bs = eps->lobpcg_bs > 0 ? eps->lobpcg_bs : std::min(16, nev);
  B200_ARG_CHECK(n >= 5 * bs, "the problem size is too small relative to the block size");
  const int kmin = std::max(3 * bs, ((nev - 1) / bs + 3) * bs);
  int ncv = eps->ncv;
  if (ncv > 0) B200_ARG_CHECK(ncv >= kmin, "the value of ncv is not sufficiently large");
  else ncv = kmin;
  B200_ARG_CHECK(eps->mpd <= 0 || eps->mpd == 3 * bs, "LOBPCG requires mpd = 3*blocksize");
  B200_ARG_CHECK(ncv + 2 < kMaxCols && 3 * bs + 2 < kMaxCols, "ncv too large for this build");
  const int mpd = 3 * bs;
  const int max_it = eps->max_it > 0 ? eps->max_it : std::max(100, 2 * n / ncv);
  const double tol = eps->tol > 0.0 ? eps->tol : 1e-8;
  const double restart = eps->lobpcg_restart > 0.0 ? eps->lobpcg_restart : 0.9;
  const int guard = bs == 1 ? 0 : std::min((int)((1.0 - restart) * bs + 0.45), bs - 1);
  const bool lock = eps->lobpcg_lock != 0;
  const bool flip = eps->which == B200_LARGEST_REAL;
  const bool useY = nev > bs - guard;
  eps->n_ = n;
  eps->ncv_ = ncv;
  eps->mpd_ = mpd;
  eps->max_it_ = max_it;
  eps->tol_ = tol;
  memset(&eps->stats, 0, sizeof(eps->stats));
  const uint64_t launches0 = launch_count();
  // Optional phase timing (b200_eps_set_timing): host clock between stream synchronisations at the
  // edges of each phase.  ms_spmv: BVMatMult; ms_orth: BVOrthogonalize and BVOrthogonalizeVec of
  // the blocks; ms_restart: the Rayleigh-Ritz projections (BVDot, DSSolve, BVMult); ms_total: all.
  using clk = std::chrono::steady_clock;
  const bool timing = eps->timing != 0;
  auto phase_begin = [&]() {
    if (timing) cudaStreamSynchronize(eps->stream);
    return clk::now();
  };
  auto phase_end = [&](clk::time_point t0, double &acc) {
    if (!timing) return;
    cudaStreamSynchronize(eps->stream);
    acc += std::chrono::duration<double, std::milli>(clk::now() - t0).count();
  };
  const clk::time_point t_solve = phase_begin();

  // EPSAllocateSolution(eps,0): V with ncv columns
  if (eps->V) {
    int bn, bm, bld;
    b200_bv_get_sizes(eps->V, &bn, &bm, &bld);
    if (bn != n || bm != ncv || eps->V->stream != eps->stream) {
      b200_bv_destroy(eps->V);
      eps->V = nullptr;
    }
  }
  if (!eps->V) B200_CHECK(b200_bv_create(n, ncv, eps->stream, &eps->V));
  b200_bv V = eps->V;
  if (!eps->resid_buf) B200_CUDA_CHECK(dev_malloc(&eps->resid_buf, sizeof(double) * 8));
  B200_CUDA_CHECK(cudaMemsetAsync(V->V, 0, sizeof(double) * V->ld * (size_t)(V->m + 1), V->stream));
  V->nrand = 0;
  Blocks B;
  B200_CHECK(b200_bv_create(n, 3 * bs, eps->stream, &B.Z));
  B200_CHECK(b200_bv_create(n, bs, eps->stream, &B.X));
  B200_CHECK(b200_bv_create(n, bs, eps->stream, &B.R));
  B200_CHECK(b200_bv_create(n, bs, eps->stream, &B.P));
  B200_CHECK(b200_bv_create(n, bs, eps->stream, &B.AX));
  B200_CHECK(b200_bv_create(n, useY ? nev : 1, eps->stream, &B.Y));
  B200_CHECK(b200_bv_create(n, 3 * bs, eps->stream, &B.W));  // A Z of BVMatProject
  for (b200_bv b : {B.Z, B.X, B.R, B.P, B.AX, B.Y, B.W})
    B200_CUDA_CHECK(cudaMemsetAsync(b->V, 0, sizeof(double) * b->ld * (size_t)(b->m + 1), b->stream));
  // the blocks are BVDuplicateResize copies of eps->V and inherit its orthogonalization settings
  // (BVDuplicate_Private, bvbasic.c:1619-1632)
  V->orthog_block = eps->orthog_block;
  for (b200_bv b : {B.Z, B.X, B.R, B.P, B.AX, B.Y, B.W}) b->orthog_block = eps->orthog_block;
  b200_bv Z = B.Z, X = B.X, R = B.R, P = B.P, AX = B.AX, Y = B.Y, W = B.W;
  active(Y, 0, 0);
  if (eps->pc == B200_PC_JACOBI) {
    B200_ARG_CHECK(A->kind == kMatCsr && !A->a.f32, "the Jacobi preconditioner needs an FP64 CSR operator");
    if (eps->dinv_of != (const void *)A) {
      dev_free(eps->dinv);
      eps->dinv = nullptr;
      B200_CUDA_CHECK(dev_malloc(&eps->dinv, sizeof(double) * (size_t)n));
      B200_CUDA_CHECK(inverse_diagonal_launch(n, A->a.rowptr, A->a.colind, static_cast<const double *>(A->a.vals),
                                              eps->dinv, eps->stream));
      eps->dinv_of = A;
    }
  }

  eps->eigr.assign(ncv + 3 * bs, 0.0);
  eps->errest.assign(ncv + 3 * bs, 0.0);
  eps->perm.assign(ncv + 3 * bs, 0);
  eps->nconv = 0;
  eps->its = 0;
  eps->reason = B200_CONVERGED_ITERATING;
  eps->solved = false;
  std::vector<double> MA((size_t)mpd * mpd), MB((size_t)mpd * mpd), Q((size_t)mpd * mpd), wr(mpd);
  std::vector<double> &eigr = eps->eigr, &errest = eps->errest;

  // EPSSetUp: the initial space; 2-3: more initial vectors
  active(V, 0, ncv);
  B200_CHECK(eps_insert_initial_space(eps, V, ncv));
  for (int k = eps->nini_eff; k < ncv - bs; ++k) {
    B200_CUDA_CHECK(random_launch(col(V, k), n, V->seed, V->nrand++, V->stream));
    double nrm = 0.0;
    B200_CHECK(bv_orth_column(V, k, 1, nullptr, &nrm, nullptr));
  }
  int nv = bs, locked = 0, nconv = 0, its = 0, reason = B200_CONVERGED_ITERATING, eps_its = 0, eps_nconv = 0;
  active(V, 0, nv);
  active(Z, 0, nv);
  B200_CUDA_CHECK(bv_copy(V, Z));
  B200_CUDA_CHECK(bv_copy(Z, X));

  // 4. Rayleigh-Ritz on X alone (also after hard locking)
  auto rayleigh_ritz_x = [&]() -> b200_status {
    clk::time_point t0 = phase_begin();
    B200_CHECK(bv_mat_mult(X, A, AX));
    phase_end(t0, eps->stats.ms_spmv);
    eps->stats.lanczos_steps += X->k - X->l;
    t0 = phase_begin();
    std::fill(MA.begin(), MA.end(), 0.0);
    B200_CHECK(b200_bv_dot(AX, X, MA.data(), mpd));  // BVMatProject(AX,NULL,X,M): M = X^T AX
    if (flip)
      for (double &v : MA) v = -v;
    std::fill(MB.begin(), MB.end(), 0.0);
    for (int i = 0; i < nv; ++i) MB[i + (size_t)i * mpd] = 1.0;
    B200_CHECK(ds_ghep(nv, mpd, MA, MB, wr, Q));
    for (int j = 0; j < nv; ++j)
      if (locked + j < ncv) eigr[locked + j] = flip ? -wr[j] : wr[j];
    B200_CHECK(b200_bv_mult_inplace(X, Q.data(), mpd, 0, nv));
    B200_CHECK(b200_bv_mult_inplace(AX, Q.data(), mpd, 0, nv));
    phase_end(t0, eps->stats.ms_restart);
    return B200_OK;
  };
  B200_CHECK(rayleigh_ritz_x());

  // 6. main loop
  while (reason == B200_CONVERGED_ITERATING) {
    if (lock) {
      active(R, nconv, bs);
      active(AX, nconv, bs);
    }
    // 7. residuals R = AX - X diag(eigr)
    int ini = lock ? nconv : 0;
    if (AX->l == ini && AX->k == bs && R->l == ini && R->k == bs) {  // BVCopy + VecAXPY per column, one launch
      B200_CUDA_CHECK(resid_block_launch(col(R, ini), R->ld, col(AX, ini), AX->ld, col(X, ini), X->ld, n, bs - ini,
                                         eigr.data() + locked + ini, R->stream));
    } else {
      B200_CUDA_CHECK(bv_copy(AX, R));
      for (int j = ini; j < bs; ++j) B200_CUDA_CHECK(axmy_launch(col(R, j), col(X, j), eigr[locked + j], n, R->stream));
    }
    // 8. residual norms and the active set
    int k = ini;
    bool countc = true;
    std::vector<double> rnorm(bs);
    active(R, ini, bs);
    B200_CHECK(bv_column_norms(R, rnorm.data()));  // all residual norms, one synchronisation
    for (int j = ini; j < bs; ++j) {
      const int i = locked + j;
      const double nrm = rnorm[j - ini];
      errest[i] = (eigr[i] != 0.0) ? nrm / std::fabs(eigr[i]) : 1.7976931348623157e308;
      if (countc) {
        if (errest[i] < tol) ++k;
        else countc = false;
      }
      if (!countc) break;
    }
    nconv = k;
    eps_nconv = locked + nconv;
    if (eps_nconv >= nev) reason = B200_CONVERGED_TOL;  // EPSStoppingBasic
    else if (eps_its + its >= max_it) reason = B200_DIVERGED_ITS;
    if (reason != B200_CONVERGED_ITERATING || nconv >= bs - guard) {
      active(V, locked, eps_nconv);
      active(X, 0, nconv);
      B200_CUDA_CHECK(bv_copy(X, V));
    }
    if (reason != B200_CONVERGED_ITERATING) break;
    if (nconv >= bs - guard) {
      eps_its += its - 1;
      its = 0;
    } else {
      ++its;
    }

    if (nconv >= bs - guard) {  // hard locking and new initial vectors
      active(Y, locked, locked + nconv);
      B200_CUDA_CHECK(bv_copy(X, Y));
      active(Y, 0, locked + nconv);
      for (int j = nconv; j < bs; ++j) {
        B200_CUDA_CHECK(bv_copy_column(X, j, j - nconv));
        B200_CUDA_CHECK(bv_copy_column(R, j, j - nconv));
        B200_CUDA_CHECK(bv_copy_column(P, j, j - nconv));
        B200_CUDA_CHECK(bv_copy_column(AX, j, j - nconv));
      }
      active(V, locked + bs, locked + bs + nconv);
      active(X, bs - nconv, bs);
      B200_CUDA_CHECK(bv_copy(V, X));
      const clk::time_point t0 = phase_begin();
      {
        std::vector<double *> vs;
        for (int j = bs - nconv; j < bs; ++j) vs.push_back(col(X, j));
        int bd = 0;
        B200_CHECK(bv_orthonormalize_vecs(Y, vs.data(), (int)vs.size(), &bd));
        if (bd) reason = B200_DIVERGED_BREAKDOWN;
      }
      if (reason != B200_CONVERGED_ITERATING) break;
      locked += nconv;
      nconv = 0;
      active(X, nconv, bs);
      B200_CHECK(b200_bv_orthogonalize(X, nullptr, 0));
      phase_end(t0, eps->stats.ms_orth);
      active(Z, nconv, bs);
      active(AX, nconv, bs);
      B200_CUDA_CHECK(bv_copy(X, Z));
      nv = bs;
      B200_CHECK(rayleigh_ritz_x());
      continue;
    }

    ini = lock ? nconv : 0;
    if (lock) {
      active(R, nconv, bs);
      active(P, nconv, bs);
      active(AX, nconv, bs);
    }
    // 9. preconditioner on the residuals, then against the locked vectors
    if (eps->pc == B200_PC_JACOBI)
      B200_CUDA_CHECK(diag_scale_launch(col(R, ini), R->ld, n, bs - ini, eps->dinv, R->stream));
    clk::time_point t0 = phase_begin();
    if (locked > 0) {
      std::vector<double *> vs;
      for (int j = ini; j < bs; ++j) vs.push_back(col(R, j));
      int bd = 0;
      B200_CHECK(bv_orthonormalize_vecs(Y, vs.data(), (int)vs.size(), &bd));
      if (bd) {
        reason = B200_DIVERGED_BREAKDOWN;
        break;
      }
    }
    // 11. orthonormalise the preconditioned residuals; 13-16 the conjugate directions
    if (its > 1) {
      B200_CHECK(bv_orthogonalize_pair(R, P));  // independent blocks: one host round trip for both
    } else {
      B200_CHECK(b200_bv_orthogonalize(R, nullptr, 0));
    }
    phase_end(t0, eps->stats.ms_orth);
    // 17-23. Z = [X R P] and the Gram matrices Z^T A Z, Z^T Z
    active(Z, 0, bs);
    active(X, 0, bs);
    B200_CUDA_CHECK(bv_copy(X, Z));
    active(Z, bs, 2 * bs - ini);
    B200_CUDA_CHECK(bv_copy(R, Z));
    if (its > 1) {
      active(Z, 2 * bs - ini, 3 * bs - 2 * ini);
      B200_CUDA_CHECK(bv_copy(P, Z));
    }
    nv = its > 1 ? 3 * bs - 2 * ini : 2 * bs - ini;
    active(Z, 0, nv);
    active(W, 0, nv);
    t0 = phase_begin();
    B200_CHECK(bv_mat_mult(Z, A, W));  // BVMatProject_MatMult: W = A Z, M = Z^T W
    phase_end(t0, eps->stats.ms_spmv);
    eps->stats.lanczos_steps += nv;
    t0 = phase_begin();
    std::fill(MA.begin(), MA.end(), 0.0);
    std::fill(MB.begin(), MB.end(), 0.0);
    // BVMatProject's M = Z^T W and BVDot's Z^T Z, one pass over both blocks
    B200_CHECK(bv_dot_pair(W, Z, MA.data(), MB.data(), mpd));
    if (flip)
      for (double &v : MA) v = -v;
    // 24. the projected pencil
    B200_CHECK(ds_ghep(nv, mpd, MA, MB, wr, Q));
    for (int j = 0; j < nv; ++j)
      if (locked + j < ncv) eigr[locked + j] = flip ? -wr[j] : wr[j];
    // 25-33. Ritz vectors and the new conjugate directions
    active(Z, bs, nv);
    if (lock) active(P, 0, bs);
    B200_CHECK(b200_bv_mult(P, 1.0, 0.0, Z, Q.data(), mpd));
    active(X, 0, bs);
    B200_CUDA_CHECK(bv_copy(P, X));
    if (lock) active(P, nconv, bs);
    active(Z, 0, bs);
    B200_CHECK(b200_bv_mult(X, 1.0, 1.0, Z, Q.data(), mpd));
    phase_end(t0, eps->stats.ms_restart);
    if (lock) active(X, nconv, bs);
    t0 = phase_begin();
    B200_CHECK(bv_mat_mult(X, A, AX));
    phase_end(t0, eps->stats.ms_spmv);
    eps->stats.lanczos_steps += X->k - X->l;
  }
  eps_its += its;

  // EPSSolve post-processing: SlepcSortEigenvalues (slepcsc.c:89-149)
  eps->nconv = eps_nconv;
  eps->its = eps_its;
  eps->reason = reason;
  auto sc = [&](double a, double b) {
    if (eps->which == B200_SMALLEST_REAL) return (a > b) ? 1 : (a < b) ? -1 : 0;
    return (a < b) ? 1 : (a > b) ? -1 : 0;
  };
  std::vector<int> &perm = eps->perm;
  for (int i = 0; i < eps_nconv; ++i) perm[i] = i;
  for (int i = eps_nconv - 1; i >= 0; --i) {
    const double re = eigr[perm[i]];
    int j = i + 1;
    while (j < eps_nconv) {
      if (sc(re, eigr[perm[j]]) <= 0) break;
      std::swap(perm[j - 1], perm[j]);
      ++j;
    }
  }
  active(V, 0, eps_nconv);
  B200_CUDA_CHECK(cudaStreamSynchronize(eps->stream));
  phase_end(t_solve, eps->stats.ms_total);
  eps->stats.restarts = eps_its;
  eps->stats.kernel_launches = (int64_t)(launch_count() - launches0);
  eps->solved = true;
  return B200_OK;
}
