// Mixed-precision Krylov-Schur (b200_eps_set_precision(B200_PRECISION_MIXED)).
//
// No SLEPc counterpart: SLEPc runs EPSSolve in the one precision PETSc was
// configured with.  The plain path (lib.cu) restates EPSSolve_KrylovSchur_Default
// (src/eps/impls/krylov/krylovschur/krylovschur.c:227-348) in FP64; this form
// keeps its restart loop and changes where the bytes go:
//
//  Phase 1 -- the same thick-restart loop (Lanczos with CGS + DGKS "if
//  needed", DSHEP on the host, locking, keep = 0.5) with the basis stored in
//  FP32 and the matrix values in FP32.  The SpMV reads an FP32 column, every
//  product and sum is FP64, the vector being orthogonalised stays FP64 until
//  it is normalised, and only then is it rounded into the FP32 basis.  The
//  Gram-Schmidt passes, the SpMV and the restart move half the bytes of the
//  FP64 basis.  The loop stops at a loose tolerance (tol_low): the rounding
//  of the stored basis (about 6e-8 relative) bounds the residuals this phase
//  can reach.
//
//  Phase 2 -- FP64 refinement of the block of the nev + guard leading Ritz
//  vectors (taken from the last projected problem, so the block holds
//  eigenvectors not yet converged as well): sweeps of a Chebyshev filter of
//  degree d that damps [a, b] (the spectrum bound from the Gershgorin discs
//  to the weakest Ritz value of the block) and amplifies the wanted end
//  (Zhou and Saad, SIAM J. Matrix Anal. Appl. 29 (2007), the scaled
//  three-term recurrence), then CholQR2 (Gram matrix on the device, Cholesky
//  on the host, twice) and an FP64 Rayleigh-Ritz step (block SpMV, Q^T A Q,
//  host dsyevd).  The sweeps stop when every wanted residual
//  ||A x - theta x|| / |theta|, computed in FP64 with the FP64 matrix,
//  is below tol.  A block method also recovers copies of repeated eigenvalues
//  that a single-vector Krylov run can miss.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <initializer_list>
#include <vector>

#include "common.h"
#include "internal.h"
#include "kernels.h"
#include "objects.h"

extern "C" void scipy_dpotrf_(const char *uplo, const int *n, double *a, const int *lda, int *info, size_t);
extern "C" void scipy_dtrtri_(const char *uplo, const char *diag, const int *n, double *a, const int *lda, int *info,
                              size_t, size_t);
extern "C" void scipy_dsyevd_(const char *jobz, const char *uplo, const int *n, double *a, const int *lda, double *w,
                              double *work, const int *lwork, int *iwork, const int *liwork, int *info, size_t,
                              size_t);

using namespace b200;

namespace {

constexpr double kDefaultTolLow = 1e-6;
constexpr int kDefaultDegree = 128;
constexpr int kDefaultMaxSweeps = 40;
constexpr int kMaxBlock = 128;  // columns of the refinement block (row-panel GEMM limit)
constexpr int kBlocks = 5;      // FP64 blocks of the refinement phase

template <typename T>
b200_status ensure(T **p, size_t *cap, size_t count) {
  if (*cap >= count && *p) return B200_OK;
  cudaFree(*p);
  *p = nullptr;
  *cap = 0;
  if (cudaMalloc(p, sizeof(T) * (count ? count : 1)) != cudaSuccess) {
    *p = nullptr;
    b200_set_last_error(__FILE__, __LINE__, "cudaMalloc failed for the mixed-precision buffers");
    return B200_ERR_NOMEM;
  }
  *cap = count;
  return B200_OK;
}

struct Mixed {
  b200_eps eps;
  b200_bv V;  // the FP64 BV of the solver: Gram-Schmidt work arrays, T, and the final eigenvectors
  cudaStream_t s;
  int n, ncv, ld32;
  float *V32;
  double *wv;

  std::vector<cudaEvent_t> ev;  // per-step SpMV / Gram-Schmidt events when timing is on
  double ms_spmv = 0.0, ms_orth = 0.0;

  float *col32(int j) const { return V32 + (size_t)j * ld32; }
  void release_events() {
    for (auto e : ev) cudaEventDestroy(e);
    ev.clear();
  }
  ~Mixed() { release_events(); }

  GsPassArgs args(int jb, int step, double *T) const {
    GsPassArgs a{};
    a.V = nullptr;
    a.ld = 0;
    a.V32 = V32;
    a.ld32 = ld32;
    a.wvec = wv;
    a.total_cols = ncv + 1;
    a.n = n;
    a.jb = jb;
    a.wcol = jb;
    a.hacc = V->coefbuf + (size_t)jb * V->ldc;
    a.T = T;
    a.ldt = V->ldt;
    a.step = step;
    a.normalize = 1;
    a.column = 1;
    a.fast32 = eps->mixed_fp32_pass;
    return a;
  }

  // EPSGetStartVector (epssolve.c:841-870) on the FP32 basis: column i from the initial vector
  // (i == 0 and one was given) or the random stream, orthonormalised in FP64, then rounded.
  b200_status start_vector(int i, int *breakdown) {
    if (i > 0 || eps->nini_eff == 0) B200_CUDA_CHECK(random_launch(wv, n, V->seed, V->nrand++, s));
    else B200_CUDA_CHECK(copy_launch(wv, col(V, 0), n, s));
    B200_CUDA_CHECK(gs_state_reset(V->gs, V->eta, s));
    GsPassArgs a = args(i, -1, nullptr);
    B200_CUDA_CHECK(gs_orthogonalize_launch(a, V->gs, s));
    GsState st;
    B200_CHECK(bv_state(V, &st));
    const bool bad = st.lindep || st.beta_out == 0.0;
    if (breakdown) *breakdown = bad;
    else if (bad) {
      b200_set_last_error(__FILE__, __LINE__,
                          i ? "unable to generate more start vectors" : "initial vector is zero or in the deflation space");
      return B200_ERR_BREAKDOWN;
    }
    B200_CUDA_CHECK(to_f32_launch(col32(i), wv, n, s));
    return B200_OK;
  }

  // BVMatLanczos on the FP32 basis: steps k..m-1 back to back, one synchronisation at the end.
  b200_status lanczos(int k, int *m, double *alpha, double *beta_h, double *beta, int *breakdown, GsState *st_out) {
    const int m0 = *m;
    const bool timing = eps->timing != 0;
    if (timing)
      while (ev.size() < (size_t)3 * (m0 - k)) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) break;
        ev.push_back(e);
      }
    const bool have_ev = timing && ev.size() >= (size_t)3 * (m0 - k);
    B200_CUDA_CHECK(gs_state_reset(V->gs, eps->mixed_eta1 >= 0.0 ? eps->mixed_eta1 : V->eta, s));
    for (int j = k; j < m0; ++j) {
      const size_t e = (size_t)3 * (j - k);
      if (have_ev) cudaEventRecord(ev[e], s);
      B200_CUDA_CHECK(mat_spmv_x32(eps->A, col32(j), wv, s, V->gs.st, j));
      if (have_ev) cudaEventRecord(ev[e + 1], s);
      GsPassArgs a = args(j + 1, j, V->T);
      B200_CUDA_CHECK(gs_orthogonalize_launch(a, V->gs, s));
      B200_CUDA_CHECK(to_f32_launch(col32(j + 1), wv, n, s));
      if (have_ev) cudaEventRecord(ev[e + 2], s);
    }
    double *hT = V->hpin + 64;
    B200_CUDA_CHECK(cudaMemcpyAsync(hT, V->T, sizeof(double) * 2 * (size_t)V->ldt, cudaMemcpyDeviceToHost, s));
    GsState st;
    B200_CHECK(bv_state(V, &st));
    *st_out = st;
    int mm = m0, bd = 0;
    if (st.halt) {
      mm = st.halt_step + 1;
      bd = 1;
    }
    for (int j = k; j < mm; ++j) {
      alpha[j] = hT[j];
      beta_h[j] = hT[V->ldt + j];
    }
    *m = mm;
    *beta = st.beta_out;
    *breakdown = bd;
    if (have_ev)
      for (int j = k; j < m0; ++j) {
        const size_t e = (size_t)3 * (j - k);
        float t = 0.f;
        if (cudaEventElapsedTime(&t, ev[e], ev[e + 1]) == cudaSuccess) ms_spmv += t;
        if (cudaEventElapsedTime(&t, ev[e + 1], ev[e + 2]) == cudaSuccess) ms_orth += t;
      }
    return B200_OK;
  }
};

// Order of the refinement block: indices of theta sorted by the wanted end (DsHep::compare).
std::vector<int> wanted_order(int which, const std::vector<double> &theta) {
  std::vector<int> idx(theta.size());
  for (size_t i = 0; i < idx.size(); ++i) idx[i] = (int)i;
  std::stable_sort(idx.begin(), idx.end(),
                   [&](int x, int y) { return DsHep::compare(which, theta[x], theta[y]) < 0; });
  return idx;
}

}  // namespace

b200_status b200::mixed_solve(b200_eps eps) {
  const int which = eps->which;
  B200_ARG_CHECK(which == B200_LARGEST_REAL || which == B200_SMALLEST_REAL || which == B200_LARGEST_MAGNITUDE,
                 "the mixed-precision solver needs which = largest real, smallest real or largest magnitude");
  b200_bv V = eps->V;
  cudaStream_t s = eps->stream;
  const int n = eps->n_, ncv = eps->ncv_, mpd = eps->mpd_, nev = eps->nev;
  const double tol = eps->tol_;
  const double tol_low = std::max(tol, eps->mixed_tol_low > 0.0 ? eps->mixed_tol_low : kDefaultTolLow);
  const int degree = eps->mixed_degree > 0 ? eps->mixed_degree : kDefaultDegree;
  const int guard = eps->mixed_guard >= 0 ? eps->mixed_guard : std::max(8, nev / 2);
  const int max_sweeps = eps->mixed_max_sweeps > 0 ? eps->mixed_max_sweeps : kDefaultMaxSweeps;
  B200_CHECK(mat_mixed_prepare(eps->A, s));

  Mixed M{};
  M.eps = eps;
  M.V = V;
  M.s = s;
  M.n = n;
  M.ncv = ncv;
  M.ld32 = (n + 31) / 32 * 32;
  B200_CHECK(ensure(&eps->V32, &eps->V32_cap, (size_t)M.ld32 * (ncv + 1)));
  B200_CHECK(ensure(&eps->wv, &eps->wv_cap, (size_t)n + 2));
  B200_CUDA_CHECK(cudaMemsetAsync(eps->wv, 0, sizeof(double) * ((size_t)n + 2), s));
  M.V32 = eps->V32;
  M.wv = eps->wv;
  const int sms = num_sms_host();
  const size_t work_len = (size_t)sms * kMaxBlock * kMaxBlock;
  // mred: Q of the restart / block build ((ncv+1)^2), G/W (kMaxBlock^2 each), theta, norms, bounds, reductions
  const size_t q_len = (size_t)(ncv + 1) * (ncv + 1), sq = (size_t)kMaxBlock * kMaxBlock;
  B200_CHECK(ensure(&eps->mred, &eps->mred_cap, q_len + 2 * sq + 3 * kMaxBlock + 8 + work_len));
  double *Qdev = eps->mred, *Gdev = Qdev + q_len, *Wdev = Gdev + sq, *thdev = Wdev + sq;
  double *nrmdev = thdev + kMaxBlock, *bnddev = nrmdev + 2 * kMaxBlock, *work = bnddev + 8;

  DsHep &ds = eps->ds;
  memset(&eps->stats, 0, sizeof(eps->stats));
  const uint64_t launches0 = launch_count();
  cudaEvent_t t0 = nullptr, t1 = nullptr, t2 = nullptr;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  cudaEventCreate(&t2);
  cudaEventRecord(t0, s);

  // ---------------------------------------------------------------- phase 1
  eps->nconv = 0;
  eps->its = 0;
  eps->reason = B200_CONVERGED_ITERATING;
  eps->solved = false;
  V->nrand = 0;
  b200_bv_set_active_columns(V, 0, V->m);
  B200_CHECK(eps_insert_initial_space(eps, V, ncv));
  B200_CHECK(M.start_vector(0, nullptr));
  int l = 0, nv = 0, nconv = 0;
  double beta = 0.0;
  int reason = B200_CONVERGED_ITERATING;
  std::vector<double> hq;
  while (reason == B200_CONVERGED_ITERATING) {
    eps->its++;
    nv = std::min(nconv + mpd, ncv);
    ds.set_dimensions(nv, nconv, nconv + l);
    int breakdown = 0;
    GsState st{};
    B200_CHECK(M.lanczos(nconv + l, &nv, ds.d(), ds.e(), &beta, &breakdown, &st));
    eps->stats.lanczos_steps += nv - (nconv + l);
    for (int j = nconv + l; j < nv; ++j) eps->stats.column_visits += j + 2;
    eps->stats.gs_passes += st.passes;
    eps->stats.gs_bytes += (int64_t)st.bytes;
    ds.set_dimensions(nv, nconv, nconv + l);
    ds.set_state(l ? DsHep::kRaw : DsHep::kIntermediate);
    B200_CHECK(ds.solve(eps->eigr.data()));
    ds.sort(eps->eigr.data());
    ds.update_extra_row();
    int k = nv;
    for (int kk = nconv; kk < nv; ++kk) {
      const double re = eps->eigr[kk];
      const double resnorm = std::fabs(ds.Q()[ds.n() - 1 + (size_t)kk * ds.ld()]) * beta;
      const double w = std::fabs(re);
      eps->errest[kk] = (w != 0.0) ? resnorm / w : 1.79769313486231571e+308;
      if (eps->errest[kk] >= tol_low) {
        k = kk;
        break;
      }
    }
    if (k >= nev) reason = B200_CONVERGED_TOL;
    else if (eps->its >= eps->max_it_) reason = B200_DIVERGED_ITS;
    else if (eps->max_restarts > 0 && eps->stats.restarts + 1 >= eps->max_restarts) reason = B200_DIVERGED_ITS;
    if (reason != B200_CONVERGED_ITERATING) break;  // the block is built from this projected problem
    l = (breakdown || k == nv) ? 0 : std::max(1, (int)((nv - k) * eps->keep));
    if (breakdown || k == nv) {
      if (k < nev) {
        int bd = 0;
        B200_CHECK(M.start_vector(k, &bd));
        if (bd) reason = B200_DIVERGED_BREAKDOWN;
      }
    } else {
      ds.truncate(k + l);
    }
    // BVMultInPlace(V, Q, nconv, k+l) on the FP32 basis
    const int kq = nv - nconv, nc = k + l - nconv;
    if (nc > 0 && kq > 0) {
      hq.assign((size_t)kq * nc, 0.0);
      for (int j = 0; j < nc; ++j)
        memcpy(hq.data() + (size_t)j * kq, ds.Q() + (size_t)nconv + (size_t)(nconv + j) * ds.ld(),
               sizeof(double) * kq);
      B200_CUDA_CHECK(cudaMemcpyAsync(Qdev, hq.data(), sizeof(double) * hq.size(), cudaMemcpyHostToDevice, s));
      B200_CUDA_CHECK(multinplace_launch_f32(M.V32, M.ld32, n, nconv, nv, Qdev, kq, nconv, k + l, s));
    }
    if (reason == B200_CONVERGED_ITERATING && !breakdown)
      B200_CUDA_CHECK(
          cudaMemcpyAsync(M.col32(k + l), M.col32(nv), sizeof(float) * n, cudaMemcpyDeviceToDevice, s));
    nconv = k;
    eps->stats.restarts++;
  }
  eps->stats.phase1_restarts = eps->stats.restarts;
  eps->stats.ms_spmv = M.ms_spmv;
  eps->stats.ms_orth = M.ms_orth;  // Gram-Schmidt passes and the FP32 store of each new column
  M.release_events();
  cudaEventRecord(t1, s);
  if (reason == B200_DIVERGED_BREAKDOWN || nv <= 0) {
    B200_CUDA_CHECK(cudaStreamSynchronize(s));
    eps->nconv = 0;
    eps->reason = reason;
    eps->solved = true;
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    cudaEventDestroy(t2);
    return B200_OK;
  }

  // ---------------------------------------------------------------- phase 2
  // The block: X = V32(:, 0:nv) Qb with Qb = [I 0; 0 Q(nconv:nv, nconv:kb)], FP64 result.
  const int kb = std::min(std::min(nev + guard, nv), kMaxBlock);
  B200_ARG_CHECK(kb >= nev, "the refinement block cannot hold nev vectors (ncv too small for the mixed solver)");
  const int ldb = (n + 31) / 32 * 32;
  B200_CHECK(ensure(&eps->blk, &eps->blk_cap, (size_t)kBlocks * ldb * kb));
  double *B[kBlocks];
  for (int i = 0; i < kBlocks; ++i) B[i] = eps->blk + (size_t)i * ldb * kb;
  {
    hq.assign((size_t)nv * kb, 0.0);
    for (int c = 0; c < kb; ++c) {
      if (c < nconv) hq[(size_t)c * nv + c] = 1.0;
      else
        for (int r = nconv; r < nv; ++r) hq[(size_t)c * nv + r] = ds.Q()[(size_t)r + (size_t)c * ds.ld()];
    }
    B200_CUDA_CHECK(cudaMemcpyAsync(Qdev, hq.data(), sizeof(double) * hq.size(), cudaMemcpyHostToDevice, s));
    B200_CUDA_CHECK(panel_mult_launch_f32(B[0], ldb, M.V32, M.ld32, n, nv, kb, Qdev, nv, s));
  }
  std::vector<double> theta(eps->eigr.begin(), eps->eigr.begin() + kb);
  B200_CUDA_CHECK(mat_gershgorin(eps->A, bnddev, work, (int)std::min(work_len, (size_t)1 << 30), s));
  double bounds[2];
  B200_CUDA_CHECK(cudaMemcpyAsync(bounds, bnddev, sizeof(bounds), cudaMemcpyDeviceToHost, s));
  B200_CUDA_CHECK(cudaStreamSynchronize(s));

  int x = 0;  // block index of X
  std::vector<double> G((size_t)kb * kb), Wm((size_t)kb * kb), rel(kb, 0.0), nrm(kb);
  int lwork = 1 + 6 * kb + 2 * kb * kb, liwork = 3 + 5 * kb;
  std::vector<double> lw((size_t)lwork);
  std::vector<int> liw((size_t)liwork);
  int sweeps = 0, done_conv = 0, used_degree = 0, nlock = 0;
  const int wl = (int)std::min(work_len, (size_t)1 << 30);
  while (sweeps < max_sweeps) {
    ++sweeps;
    // filter interval from the current Ritz values
    std::vector<int> ord = wanted_order(which, theta);
    const double best = theta[ord[0]], worst = theta[ord[kb - 1]];
    double a, b;
    if (which == B200_LARGEST_REAL) {
      a = bounds[0];
      b = worst;
    } else if (which == B200_SMALLEST_REAL) {
      a = worst;
      b = bounds[1];
    } else {
      a = -std::fabs(worst);
      b = std::fabs(worst);
    }
    const double e = 0.5 * (b - a), c = 0.5 * (b + a);
    int f = x;  // block holding the filtered vectors
    // The scaled filter maps the best Ritz value to 1 and the damped interval into [-1/T, 1/T] with
    // T = T_d(t_best): the block's condition number grows like T, so d is capped to keep T <= 1e6
    // (Cholesky QR twice is accurate in FP64 below about 1e8).
    int d = degree;
    const double tb = std::fabs((best - c) / e);
    if (tb > 1.0 && std::isfinite(tb)) {
      const double cap = std::acosh(1e6) / std::acosh(tb);
      if (cap < d) d = std::max(2, (int)cap);
    }
    used_degree = std::max(used_degree, d);
    // soft locking: the leading pairs that have converged keep their vectors; only columns
    // nlock..kb-1 are filtered (CholQR2 and Rayleigh-Ritz still take the whole block)
    const int a0 = nlock, na = kb - nlock;
    if (e > 0.0 && best != c && std::isfinite(e) && d > 0 && na > 0) {
      const double sigma1 = e / (best - c);
      const size_t off = (size_t)a0 * ldb;
      int prev = x, cur = (x + 1) % kBlocks, nxt = (x + 2) % kBlocks;
      B200_CUDA_CHECK(mat_spmm(eps->A, B[prev] + off, nullptr, B[cur] + off, ldb, na, sigma1 / e, c, 0.0, s));
      double sigma = sigma1;
      for (int i = 2; i <= d; ++i) {
        const double sn = 1.0 / (2.0 / sigma1 - sigma);
        B200_CUDA_CHECK(
            mat_spmm(eps->A, B[cur] + off, B[prev] + off, B[nxt] + off, ldb, na, 2.0 * sn / e, c, sigma * sn, s));
        const int t = prev;
        prev = cur;
        cur = nxt;
        nxt = t;
        sigma = sn;
      }
      f = cur;
      if (f != x && a0 > 0)
        B200_CUDA_CHECK(cudaMemcpy2DAsync(B[f], sizeof(double) * ldb, B[x], sizeof(double) * ldb, sizeof(double) * n,
                                          a0, cudaMemcpyDeviceToDevice, s));
      eps->stats.spmm_columns += (int64_t)na * d;
    }
    auto free_block = [&](std::initializer_list<int> used) {
      for (int i = 0; i < kBlocks; ++i)
        if (std::find(used.begin(), used.end(), i) == used.end()) return i;
      return -1;
    };
    // CholQR2: F = Q R, G = F^T F = R^T R (Cholesky on the host), Q = F R^{-1}; twice
    int npass = 2;  // one more pass after a shifted one
    for (int pass = 0; pass < npass; ++pass) {
      B200_CUDA_CHECK(dot_launch(B[f], ldb, kb, B[f], ldb, kb, n, Gdev, kb, work, wl, s, 4));
      B200_CUDA_CHECK(cudaMemcpyAsync(G.data(), Gdev, sizeof(double) * G.size(), cudaMemcpyDeviceToHost, s));
      B200_CUDA_CHECK(cudaStreamSynchronize(s));
      int info = 0;
      std::vector<double> R = G;
      scipy_dpotrf_("U", &kb, R.data(), &kb, &info, 1);
      if (info != 0) {
        // shifted Cholesky QR: G + sigma I with sigma = 11 (n kb + kb (kb+1)) u trace(G)
        double tr = 0.0;
        for (int i = 0; i < kb; ++i) tr += G[(size_t)i * kb + i];
        const double shift = 11.0 * ((double)n * kb + (double)kb * (kb + 1)) * 1.1102230246251565e-16 * tr;
        R = G;
        for (int i = 0; i < kb; ++i) R[(size_t)i * kb + i] += shift;
        info = 0;
        scipy_dpotrf_("U", &kb, R.data(), &kb, &info, 1);
        if (info != 0) {
          b200_set_last_error(__FILE__, __LINE__, "Cholesky QR of the refinement block failed (rank deficient)");
          return B200_ERR_LAPACK;
        }
        if (npass == 2) npass = pass + 3;
      }
      scipy_dtrtri_("U", "N", &kb, R.data(), &kb, &info, 1, 1);
      if (info != 0) {
        b200_set_last_error(__FILE__, __LINE__, "LAPACK dtrtri failed");
        return B200_ERR_LAPACK;
      }
      for (int j = 0; j < kb; ++j)
        for (int i = j + 1; i < kb; ++i) R[(size_t)j * kb + i] = 0.0;
      B200_CUDA_CHECK(cudaMemcpyAsync(Wdev, R.data(), sizeof(double) * R.size(), cudaMemcpyHostToDevice, s));
      const int q = free_block({f});
      B200_CUDA_CHECK(panel_mult_launch(B[q], ldb, B[f], ldb, n, kb, kb, Wdev, kb, s));
      f = q;
    }
    // Rayleigh-Ritz: H = Q^T A Q, H = W diag(theta) W^T, X = Q W, AX = (A Q) W
    const int aq = free_block({f});
    B200_CUDA_CHECK(mat_spmm(eps->A, B[f], nullptr, B[aq], ldb, kb, 1.0, 0.0, 0.0, s));
    eps->stats.spmm_columns += kb;
    B200_CUDA_CHECK(dot_launch(B[aq], ldb, kb, B[f], ldb, kb, n, Gdev, kb, work, wl, s, 4));
    B200_CUDA_CHECK(cudaMemcpyAsync(G.data(), Gdev, sizeof(double) * G.size(), cudaMemcpyDeviceToHost, s));
    B200_CUDA_CHECK(cudaStreamSynchronize(s));
    for (int j = 0; j < kb; ++j)
      for (int i = 0; i < j; ++i) {
        const double v = 0.5 * (G[(size_t)j * kb + i] + G[(size_t)i * kb + j]);
        G[(size_t)j * kb + i] = G[(size_t)i * kb + j] = v;
      }
    std::vector<double> w(kb);
    int info = 0;
    scipy_dsyevd_("V", "U", &kb, G.data(), &kb, w.data(), lw.data(), &lwork, liw.data(), &liwork, &info, 1, 1);
    if (info != 0) {
      b200_set_last_error(__FILE__, __LINE__, "LAPACK dsyevd failed");
      return B200_ERR_LAPACK;
    }
    ord = wanted_order(which, w);
    for (int j = 0; j < kb; ++j) {
      theta[j] = w[ord[j]];
      memcpy(Wm.data() + (size_t)j * kb, G.data() + (size_t)ord[j] * kb, sizeof(double) * kb);
    }
    B200_CUDA_CHECK(cudaMemcpyAsync(Wdev, Wm.data(), sizeof(double) * Wm.size(), cudaMemcpyHostToDevice, s));
    B200_CUDA_CHECK(cudaMemcpyAsync(thdev, theta.data(), sizeof(double) * kb, cudaMemcpyHostToDevice, s));
    const int xn = free_block({f, aq});
    B200_CUDA_CHECK(panel_mult_launch(B[xn], ldb, B[f], ldb, n, kb, kb, Wdev, kb, s));
    const int axn = free_block({f, aq, xn});
    B200_CUDA_CHECK(panel_mult_launch(B[axn], ldb, B[aq], ldb, n, kb, kb, Wdev, kb, s));
    B200_CUDA_CHECK(colresid_launch(B[axn], B[xn], ldb, n, kb, thdev, nrmdev, work, wl, s));
    B200_CUDA_CHECK(cudaMemcpyAsync(nrm.data(), nrmdev, sizeof(double) * kb, cudaMemcpyDeviceToHost, s));
    B200_CUDA_CHECK(cudaStreamSynchronize(s));
    x = xn;
    done_conv = 0;
    for (int i = 0; i < kb; ++i) {
      const double wabs = std::fabs(theta[i]);
      rel[i] = (wabs != 0.0) ? nrm[i] / wabs : 1.79769313486231571e+308;
    }
    while (done_conv < kb && rel[done_conv] < tol) ++done_conv;  // EPSConvergedRelative, leading pairs
    if (done_conv >= nev) break;
    nlock = done_conv;
  }
  eps->stats.filter_sweeps = sweeps;
  eps->stats.filter_degree = used_degree;  // the largest degree a sweep used
  eps->stats.block_size = kb;

  // results: eigenvectors in columns 0..kb-1 of the FP64 BV, values and residuals in order
  B200_CUDA_CHECK(cudaMemcpy2DAsync(col(V, 0), sizeof(double) * V->ld, B[x], sizeof(double) * ldb,
                                    sizeof(double) * n, kb, cudaMemcpyDeviceToDevice, s));
  for (int i = 0; i <= ncv; ++i) eps->perm[i] = i;
  for (int i = 0; i < kb; ++i) {
    eps->eigr[i] = theta[i];
    eps->errest[i] = rel[i];
  }
  eps->nconv = done_conv;
  eps->its += sweeps;
  eps->reason = done_conv >= nev ? B200_CONVERGED_TOL : B200_DIVERGED_ITS;
  cudaEventRecord(t2, s);
  cudaEventSynchronize(t2);
  float ms1 = 0.f, ms2 = 0.f;
  cudaEventElapsedTime(&ms1, t0, t1);
  cudaEventElapsedTime(&ms2, t1, t2);
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  cudaEventDestroy(t2);
  eps->stats.ms_phase1 = ms1;
  eps->stats.ms_phase2 = ms2;
  eps->stats.ms_total = ms1 + ms2;
  eps->stats.kernel_launches = (int64_t)(launch_count() - launches0);
  eps->solved = true;
  return B200_OK;
}
