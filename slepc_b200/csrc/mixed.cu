// Mixed-precision Hermitian eigensolver (b200_eps_set_precision(B200_PRECISION_MIXED)).
//
// No SLEPc counterpart: SLEPc runs EPSSolve in the one precision PETSc was configured with.  The
// plain path (lib.cu) restates EPSSolve_KrylovSchur_Default in FP64; this form returns the same
// eigenpairs (every residual ||A x - theta x|| / |theta| below tol, computed in FP64 with the FP64
// matrix) by a block method whose bytes go where a B200 moves them fastest:
//
//  A block of BP vectors (BP = 64 or 128 >= nev + guard), stored row-major, is refined by
//  Chebyshev-filtered subspace iteration (Zhou and Saad, "Self-consistent-field calculations using
//  Chebyshev-filtered subspace iteration", J. Comput. Phys. 219 (2006); the scaled three-term
//  filter of Zhou and Saad, SIAM J. Matrix Anal. Appl. 29 (2007)).  Each sweep applies a degree-d
//  polynomial that damps the unwanted part of the spectrum [a, b] (from the Gershgorin bound to the
//  weakest Ritz value of the block) and amplifies the wanted end, then re-orthonormalises the block
//  and performs a Rayleigh-Ritz step.  The degree of each sweep is chosen from the current
//  residuals and Ritz values (the Chebyshev growth at the Ritz value that is furthest from its
//  target); the sweep runs in segments, each re-orthonormalised, so that the block's condition
//  number stays bounded (by 20 in FP32, where the orthonormalisation Gram matrix is TF32).
//
//  Phase 1 (FP32): the block and the matrix values are FP32; the filter's block SpMV accumulates
//  in FP32 (rowblock.cu rb_spmm_kernel).  The orthonormalisation projection X^T X runs on the
//  tensor cores (tcgen05 kind::tf32, FP32 accumulation in TMEM) and the block is rotated by the
//  inverse square root of that Gram matrix (SVQB, host dsyevd); the Rayleigh quotients X^T X and
//  X^T A X are formed in FP64 from the FP32 data and solved as a generalised problem (host dsygvd);
//  the residual norms are FP64 sums.  The phase stops at tol_low (default 5e-7) or when a sweep no
//  longer halves the largest wanted residual (the FP32 rounding floor).
//
//  One more FP32 sweep follows, sized by the Chebyshev growth for the final tolerance (progress
//  below the FP32 floor cannot be measured in FP32, only predicted).
//
//  Phase 2 (FP64): the block is widened to FP64; a short polish filter over a wide interval removes
//  the FP32 rounding noise spread over the unwanted spectrum, and further FP64 sweeps (FP64 block
//  SpMV with the FP64 matrix, FP64 Gram products, SVQB, Rayleigh-Ritz) run until every wanted
//  residual is below tol.  A block method also finds every copy of a repeated eigenvalue in the block's reach,
//  which a single-vector Krylov run finds only through rounding.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <initializer_list>
#include <vector>

#include "common.h"
#include "internal.h"
#include "kernels.h"
#include "objects.h"
#include "rowblock.h"

extern "C" void scipy_dsyevd_(const char *jobz, const char *uplo, const int *n, double *a, const int *lda, double *w,
                              double *work, const int *lwork, int *iwork, const int *liwork, int *info, size_t,
                              size_t);
extern "C" void scipy_dpotrf_(const char *uplo, const int *n, double *a, const int *lda, int *info, size_t);
extern "C" void scipy_dtrtri_(const char *uplo, const char *diag, const int *n, double *a, const int *lda, int *info,
                              size_t, size_t);
extern "C" void scipy_dsygvd_(const int *, const char *, const char *, const int *, double *, const int *, double *,
                              const int *, double *, double *, const int *, int *, const int *, int *, size_t,
                              size_t);

using namespace b200;

namespace {

constexpr double kDefaultTolLow = 5e-7;
constexpr int kDefaultDegreeCap = 400;   // largest degree of one sweep
constexpr int kMinDegree = 6;
constexpr int kDefaultMaxSweeps = 60;    // per phase
constexpr double kSegCap32 = 20.0;      // growth of the best Ritz value per filter segment, FP32 (block condition)
constexpr double kSegCap64 = 1e4;       // the same in FP64
constexpr double kWide = 0.1;           // polish interval: pulled back by this fraction
constexpr double kPolishGrowth = 300.0; // damping of the FP32 rounding noise by the polish filter
constexpr int kBufs = 4;                // row-major blocks per precision

// The blocks come from the library's stream-ordered pool (pool_alloc): a solve that follows another
// EPS's destruction -- the one-call host API creates one per call -- reuses the same gigabytes
// instead of mapping them again.
template <typename T>
b200_status ensure(T **p, size_t *cap, size_t count, cudaStream_t s) {
  if (*cap >= count && *p) return B200_OK;
  if (*p) pool_free(*p, s);
  *p = nullptr;
  *cap = 0;
  void *q = nullptr;
  if (pool_alloc(&q, sizeof(T) * (count ? count : 1), s) != cudaSuccess) {
    b200_set_last_error(__FILE__, __LINE__, "device allocation failed for the mixed-precision buffers");
    return B200_ERR_NOMEM;
  }
  *p = static_cast<T *>(q);
  *cap = count;
  return B200_OK;
}

// Order of the pairs: indices of theta sorted by the wanted end (DsHep::compare).
std::vector<int> wanted_order(int which, const std::vector<double> &theta) {
  std::vector<int> idx(theta.size());
  for (size_t i = 0; i < idx.size(); ++i) idx[i] = (int)i;
  std::stable_sort(idx.begin(), idx.end(),
                   [&](int x, int y) { return DsHep::compare(which, theta[x], theta[y]) < 0; });
  return idx;
}

struct Block {
  b200_eps eps;
  cudaStream_t s;
  int n, bp, nev, which;
  const CsrPart *P;
  // device
  float *b32[kBufs];
  double *b64[kBufs];
  double *GH, *M, *theta_d, *res_d, *work;
  float *work32;
  int *err;
  // host
  std::vector<double> G, H, Q, theta, rel;
  double bounds[2];
  int x = 0;  // index of the current block among the buffers of the phase
  bool x32 = true;
  int64_t spmm_cols = 0;
  int max_degree = 0;  // largest degree of one sweep
  int segments = 0;
  // timing mode: device time and algorithmic bytes of the filters' block SpMVs
  cudaEvent_t f0 = nullptr, f1 = nullptr;
  double filter_ms = 0.0, filter_bytes = 0.0;
  // orthonormalisations and Rayleigh-Ritz steps: counts, and in timing mode their host wall time
  // (the stream is idle when they start: a timed filter ends with a synchronisation)
  int64_t svqb_count = 0, rr_count = 0, cholqr_count = 0;
  double svqb_ms = 0.0, rr_ms = 0.0;
  double wall_ms(std::chrono::steady_clock::time_point t0) const {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }

  void *buf(int i) const { return x32 ? (void *)b32[i] : (void *)b64[i]; }
  int free_buf(std::initializer_list<int> used) const {
    for (int i = 0; i < kBufs; ++i)
      if (std::find(used.begin(), used.end(), i) == used.end()) return i;
    return -1;
  }

  cudaError_t spmm(const void *Xin, const void *Zin, void *Y, double alpha, double shift, double beta) {
    const bool vf32 = x32 ? true : P->f32;
    const void *sv = x32 ? (P->f32 ? P->sell.vals : (const void *)P->sell.vals32) : P->sell.vals;
    const void *cv = x32 ? (P->f32 ? P->vals : (const void *)P->vals32) : P->vals;
    spmm_cols += bp;
    // algorithmic bytes: every stored nonzero (value + column index) once, X once (its gathered
    // rows counted once), Z once when present, Y once
    const double vbytes = (double)P->nnz * ((vf32 ? 4.0 : 8.0) + 4.0);
    filter_bytes += vbytes + (double)n * bp * (x32 ? 4.0 : 8.0) * (Zin ? 3.0 : 2.0);
    return rb_spmm_launch(P->sell, n, P->rowptr, P->colind, cv, sv, vf32, x32, bp, Xin, Zin, Y, alpha, shift, beta, s);
  }

  // Orthonormalisation of the current block: G = X^T X (tensor cores in FP32, FP64 otherwise),
  // scaled to unit diagonal; Cholesky QR when G factors with margin, else SVQB: G = V D V^T,
  // X <- X V D^{-1/2} (directions below 1e-12 of the largest are floored, not dropped).
  b200_status svqb() {
    const auto t0 = std::chrono::steady_clock::now();
    ++svqb_count;
    b200_status st = svqb_inner();
    if (eps->timing && st == B200_OK) {
      if (cudaStreamSynchronize(s) != cudaSuccess) return B200_ERR_CUDA;
      svqb_ms += wall_ms(t0);
    }
    return st;
  }

  b200_status svqb_inner() {
    if (x32 && !eps->mixed_fp64_gram) {
      CUtensorMap tm;
      B200_CUDA_CHECK(rb_make_tmap_f32(&tm, b32[x], n, bp));
      B200_CUDA_CHECK(rb_gram_tf32_launch(tm, nullptr, n, bp, GH, work32, err, s));
    } else {
      B200_CUDA_CHECK(rb_gram2_f64_launch(buf(x), buf(x), x32, n, bp, GH, work, s));
    }
    int herr = 0;
    B200_CUDA_CHECK(cudaMemcpyAsync(G.data(), GH, sizeof(double) * bp * bp, cudaMemcpyDeviceToHost, s));
    B200_CUDA_CHECK(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, s));
    B200_CUDA_CHECK(cudaStreamSynchronize(s));
    if (herr) {
      b200_set_last_error(__FILE__, __LINE__, "the tensor-core Gram kernel reported a device-side timeout");
      return B200_ERR_DEVICE;
    }
    for (int i = 0; i < bp; ++i)
      for (int j = 0; j < i; ++j) G[(size_t)i * bp + j] = G[(size_t)j * bp + i] = 0.5 * (G[(size_t)i * bp + j] + G[(size_t)j * bp + i]);
    // scale to unit diagonal first (SVQB, Stathopoulos and Wu 2002): d_i^{-1/2} G d_j^{-1/2}
    std::vector<double> dsc(bp);
    for (int i = 0; i < bp; ++i) {
      const double g = G[(size_t)i * bp + i];
      dsc[i] = g > 0.0 && std::isfinite(g) ? 1.0 / std::sqrt(g) : 1.0;
    }
    for (int i = 0; i < bp; ++i)
      for (int j = 0; j < bp; ++j) G[(size_t)i * bp + j] *= dsc[i] * dsc[j];
    // Cholesky QR when the scaled Gram matrix factors with margin (every pivot above 1e-4, i.e. a
    // condition number below about 1e4, which the filter segments keep): X <- X D R^{-1} with
    // D R^{-1} upper triangular -- a different orthonormal basis of the same span as SVQB's, for a
    // 64 x 64 Cholesky and triangular inverse on the host instead of an eigendecomposition.
    {
      std::vector<double> R(G);
      int info = 0;
      scipy_dpotrf_("U", &bp, R.data(), &bp, &info, 1);
      bool ok = info == 0;
      for (int j = 0; ok && j < bp; ++j) ok = R[(size_t)j * bp + j] * R[(size_t)j * bp + j] > 1e-4;
      if (ok) {
        scipy_dtrtri_("U", "N", &bp, R.data(), &bp, &info, 1, 1);
        ok = info == 0;
      }
      if (ok) {
        ++cholqr_count;
        // M[k][c] = dsc[k] Rinv(k, c); Rinv column-major and upper triangular
        for (int k = 0; k < bp; ++k)
          for (int c = 0; c < bp; ++c) Q[(size_t)k * bp + c] = k <= c ? dsc[k] * R[(size_t)c * bp + k] : 0.0;
        B200_CUDA_CHECK(cudaMemcpyAsync(M, Q.data(), sizeof(double) * bp * bp, cudaMemcpyHostToDevice, s));
        const int y = free_buf({x});
        B200_CUDA_CHECK(rb_rotate_launch(buf(x), buf(y), x32, n, bp, M, s));
        x = y;
        return B200_OK;
      }
    }
    std::vector<double> w(bp);
    B200_CHECK(syevd(G.data(), w.data()));
    const double wmax = w[bp - 1] > 0.0 ? w[bp - 1] : 1.0;
    // M[k][c] = dsc[k] V[k][c] / sqrt(max(w_c, floor)); G is column-major (symmetric): V(k,c) at [c*bp+k]
    for (int k = 0; k < bp; ++k)
      for (int c = 0; c < bp; ++c)
        Q[(size_t)k * bp + c] = dsc[k] * G[(size_t)c * bp + k] / std::sqrt(std::max(w[c], 1e-12 * wmax));
    B200_CUDA_CHECK(cudaMemcpyAsync(M, Q.data(), sizeof(double) * bp * bp, cudaMemcpyHostToDevice, s));
    const int y = free_buf({x});
    B200_CUDA_CHECK(rb_rotate_launch(buf(x), buf(y), x32, n, bp, M, s));
    x = y;
    return B200_OK;
  }

  b200_status syevd(double *a, double *w) {
    int lwork = 1 + 6 * bp + 2 * bp * bp, liwork = 3 + 5 * bp, info = 0;
    std::vector<double> lw((size_t)lwork);
    std::vector<int> liw((size_t)liwork);
    scipy_dsyevd_("V", "U", &bp, a, &bp, w, lw.data(), &lwork, liw.data(), &liwork, &info, 1, 1);
    if (info != 0) {
      b200_set_last_error(__FILE__, __LINE__, "LAPACK dsyevd failed");
      return B200_ERR_LAPACK;
    }
    return B200_OK;
  }

  // Rayleigh-Ritz on the current block: W = A X, the pencil (X^T A X, X^T X) in FP64, its
  // eigenvectors Q (wanted end first), X <- X Q, W <- W Q, residual norms ||W_c - theta_c X_c||.
  int its = 0;  // sweeps so far (the monitor's iteration number)
  b200_status monitor() {
    ++its;
    if (eps->monitors.empty() && !eps->monitor_jsonl) return B200_OK;
    return eps_monitor(eps, its, leading_converged(eps->tol_), theta.data(), rel.data(), bp);
  }

  b200_status rayleigh_ritz() {
    const auto t0 = std::chrono::steady_clock::now();
    ++rr_count;
    b200_status st = rayleigh_ritz_inner();
    if (eps->timing && st == B200_OK) rr_ms += wall_ms(t0);  // ends with a synchronisation
    return st;
  }

  b200_status rayleigh_ritz_inner() {
    const int wb = free_buf({x});
    B200_CUDA_CHECK(spmm(buf(x), nullptr, buf(wb), 1.0, 0.0, 0.0));
    B200_CUDA_CHECK(rb_gram2_f64_launch(buf(x), buf(wb), x32, n, bp, GH, work, s));
    std::vector<double> gh((size_t)2 * bp * bp);
    B200_CUDA_CHECK(cudaMemcpyAsync(gh.data(), GH, sizeof(double) * gh.size(), cudaMemcpyDeviceToHost, s));
    B200_CUDA_CHECK(cudaStreamSynchronize(s));
    // row-major X^T X and X^T W; symmetric, so column-major storage of the symmetrised parts is the same
    for (int i = 0; i < bp; ++i)
      for (int j = 0; j < bp; ++j) {
        G[(size_t)i * bp + j] = 0.5 * (gh[(size_t)i * bp + j] + gh[(size_t)j * bp + i]);
        H[(size_t)i * bp + j] = 0.5 * (gh[(size_t)bp * bp + (size_t)i * bp + j] + gh[(size_t)bp * bp + (size_t)j * bp + i]);
      }
    int itype = 1, info = 0, lwork = 1 + 6 * bp + 2 * bp * bp, liwork = 3 + 5 * bp;
    std::vector<double> w(bp), lw((size_t)lwork);
    std::vector<int> liw((size_t)liwork);
    scipy_dsygvd_(&itype, "V", "U", &bp, H.data(), &bp, G.data(), &bp, w.data(), lw.data(), &lwork, liw.data(),
                  &liwork, &info, 1, 1);
    if (info != 0) {
      b200_set_last_error(__FILE__, __LINE__, "LAPACK dsygvd failed in the Rayleigh-Ritz step (block rank deficient)");
      return B200_ERR_LAPACK;
    }
    std::vector<int> ord = wanted_order(which, w);
    for (int c = 0; c < bp; ++c) {
      theta[c] = w[ord[c]];
      for (int k = 0; k < bp; ++k) Q[(size_t)k * bp + c] = H[(size_t)ord[c] * bp + k];  // eigenvector ord[c]
    }
    B200_CUDA_CHECK(cudaMemcpyAsync(M, Q.data(), sizeof(double) * bp * bp, cudaMemcpyHostToDevice, s));
    B200_CUDA_CHECK(cudaMemcpyAsync(theta_d, theta.data(), sizeof(double) * bp, cudaMemcpyHostToDevice, s));
    const int xn = free_buf({x, wb});
    B200_CUDA_CHECK(rb_rotate_launch(buf(x), buf(xn), x32, n, bp, M, s));
    const int wn = free_buf({x, wb, xn});
    B200_CUDA_CHECK(rb_rotate_launch(buf(wb), buf(wn), x32, n, bp, M, s));
    B200_CUDA_CHECK(rb_resid_launch(buf(wn), buf(xn), x32, n, bp, theta_d, res_d, work, s));
    std::vector<double> res(bp);
    B200_CUDA_CHECK(cudaMemcpyAsync(res.data(), res_d, sizeof(double) * bp, cudaMemcpyDeviceToHost, s));
    B200_CUDA_CHECK(cudaStreamSynchronize(s));
    for (int c = 0; c < bp; ++c) {
      const double a = std::fabs(theta[c]);
      rel[c] = a != 0.0 ? res[c] / a : 1.79769313486231571e+308;
    }
    x = xn;
    return B200_OK;
  }

  // Interval [a, b] the filter damps, from the Ritz values (wanted end first) and the Gershgorin bounds.
  // wide > 0 pulls the edge next to the wanted end back by that fraction of the interval: the polish
  // filter damps everything up to there much faster at the price of leaving the band next to the
  // block's weakest Ritz value undamped.
  void interval(double *a, double *b, double wide = 0.0) const {
    const double worst = theta[bp - 1];
    if (which == B200_LARGEST_REAL) {
      *a = bounds[0];
      *b = worst - wide * (worst - bounds[0]);
    } else if (which == B200_SMALLEST_REAL) {
      *a = worst + wide * (bounds[1] - worst);
      *b = bounds[1];
    } else {
      *a = -std::fabs(worst) * (1.0 - wide);
      *b = std::fabs(worst) * (1.0 - wide);
    }
  }

  // Degree of the polish filter: growth `growth` at the weakest wanted Ritz value over the wide interval.
  int polish_degree(double wide, double growth, int cap) const {
    double a, b;
    interval(&a, &b, wide);
    const double e = 0.5 * (b - a), c = 0.5 * (b + a);
    const double t = std::fabs((theta[nev - 1] - c) / e);
    if (!(e > 0.0) || !(t > 1.0) || !std::isfinite(t)) return kMinDegree;
    const int d = (int)std::ceil(std::acosh(growth) / std::acosh(t));
    return std::max(4, std::min(d, cap));
  }

  // Degree of the next sweep: enough Chebyshev growth at the slowest unconverged wanted Ritz value
  // to bring its residual to target (the sweep runs in segments, filter_segments), at most cap.
  int choose_degree(double target, int cap) const {
    double a, b;
    interval(&a, &b);
    const double e = 0.5 * (b - a), c = 0.5 * (b + a);
    if (!(e > 0.0) || !std::isfinite(e)) return kMinDegree;
    double need = kMinDegree;
    for (int i = 0; i < nev; ++i) {
      if (rel[i] <= target) continue;
      const double t = std::fabs((theta[i] - c) / e);
      if (!(t > 1.0)) continue;
      const double d = std::acosh(std::max(rel[i] / target, 1.0)) / std::acosh(t);
      need = std::max(need, 1.1 * d + 2.0);
    }
    const int d = (int)std::ceil(std::min(need, (double)cap));
    return std::max(kMinDegree, d);
  }

  // One filter application of degree d to the current block (the scaled three-term recurrence).
  b200_status filter(int d, double wide = 0.0) {
    double a, b;
    interval(&a, &b, wide);
    const double e = 0.5 * (b - a), c = 0.5 * (b + a);
    const double best = theta[0];
    if (!(e > 0.0) || best == c || !std::isfinite(e) || d < 1) return B200_OK;
    const double sigma1 = e / (best - c);
    const bool timed = eps->timing && f0 && f1;
    const double bytes0 = filter_bytes;
    if (timed) cudaEventRecord(f0, s);
    int prev = x, cur = free_buf({x}), nxt = free_buf({x, cur});
    B200_CUDA_CHECK(spmm(buf(prev), nullptr, buf(cur), sigma1 / e, c, 0.0));
    double sigma = sigma1;
    for (int i = 2; i <= d; ++i) {
      const double sn = 1.0 / (2.0 / sigma1 - sigma);
      B200_CUDA_CHECK(spmm(buf(cur), buf(prev), buf(nxt), 2.0 * sn / e, c, sigma * sn));
      const int t = prev;
      prev = cur;
      cur = nxt;
      nxt = t;
      sigma = sn;
    }
    x = cur;
    if (timed) {
      float ms = 0.f;
      cudaEventRecord(f1, s);
      if (cudaEventSynchronize(f1) == cudaSuccess && cudaEventElapsedTime(&ms, f0, f1) == cudaSuccess)
        filter_ms += ms;
    } else {
      filter_bytes = bytes0;  // bytes are reported only with their time
    }
    return B200_OK;
  }

  // A sweep of total degree D in segments whose growth of the best Ritz value stays below seg_cap,
  // each segment but the last followed by SVQB: the block's condition number stays near seg_cap, which
  // the tensor-core (TF32) Gram matrix of the FP32 phase resolves, and the FP64 Rayleigh-Ritz step
  // runs once per sweep.
  b200_status filter_segments(int D, double seg_cap, double wide = 0.0) {
    double a, b;
    interval(&a, &b, wide);
    const double e = 0.5 * (b - a), c = 0.5 * (b + a);
    const double tb = std::fabs((theta[0] - c) / e);
    int seg = D;
    if (e > 0.0 && tb > 1.0 && std::isfinite(tb)) seg = std::max(4, (int)std::floor(std::acosh(seg_cap) / std::acosh(tb)));
    for (int done = 0; done < D;) {
      const int d = std::min(seg, D - done);
      B200_CHECK(filter(d, wide));
      done += d;
      ++segments;
      if (done < D) B200_CHECK(svqb());
    }
    return B200_OK;
  }

  double max_wanted() const {
    double m = 0.0;
    for (int i = 0; i < nev; ++i) m = std::max(m, rel[i]);
    return m;
  }
  int leading_converged(double tol) const {
    int k = 0;
    while (k < bp && rel[k] < tol) ++k;
    return k;
  }
};

}  // namespace

b200_status b200::mixed_solve(b200_eps eps) {
  const int which = eps->which;
  B200_ARG_CHECK(which == B200_LARGEST_REAL || which == B200_SMALLEST_REAL || which == B200_LARGEST_MAGNITUDE,
                 "the mixed-precision solver needs which = largest real, smallest real or largest magnitude");
  b200_bv V = eps->V;
  cudaStream_t s = eps->stream;
  const int n = eps->n_, nev = eps->nev;
  const double tol = eps->tol_;
  const double tol_low = std::max(tol, eps->mixed_tol_low > 0.0 ? eps->mixed_tol_low : kDefaultTolLow);
  const int deg_cap = eps->mixed_degree > 0 ? eps->mixed_degree : kDefaultDegreeCap;
  const int guard = eps->mixed_guard >= 0 ? eps->mixed_guard : std::max(8, nev / 2);
  const int max_sweeps = eps->mixed_max_sweeps > 0 ? eps->mixed_max_sweeps : kDefaultMaxSweeps;
  const int bp = nev + guard <= 64 ? 64 : 128;
  if (nev + guard > 128) {
    b200_set_last_error(__FILE__, __LINE__, "the mixed-precision solver holds at most 128 block vectors (nev + guard)");
    return B200_ERR_SUP;
  }
  B200_ARG_CHECK(n >= 2 * bp, "the mixed-precision solver needs n >= 2 * block width (128 or 256 rows)");
  B200_CHECK(mat_mixed_prepare(eps->A, s));

  Block B{};
  B.eps = eps;
  B.s = s;
  B.n = n;
  B.bp = bp;
  B.nev = nev;
  B.which = which;
  B.P = &eps->A->a;
  const size_t blk = (size_t)n * bp;
  B200_CHECK(ensure(&eps->rb32, &eps->rb32_cap, kBufs * blk, eps->stream));
  B200_CHECK(ensure(&eps->rb64, &eps->rb64_cap, kBufs * blk, eps->stream));
  for (int i = 0; i < kBufs; ++i) {
    B.b32[i] = eps->rb32 + (size_t)i * blk;
    B.b64[i] = eps->rb64 + (size_t)i * blk;
  }
  const int ctas = rb_gram_ctas(n, bp);
  const size_t sq = (size_t)bp * bp;
  const size_t work_len = std::max((size_t)ctas * 2 * sq, (size_t)bp * 1024);
  // mred: G|H (2 bp^2), M (bp^2), theta, res, Gershgorin work and bounds, then the reduction work
  const int gw = 1 << 16;
  B200_CHECK(ensure(&eps->mred, &eps->mred_cap, 3 * sq + 2 * (size_t)bp + 8 + gw + work_len + (size_t)ctas * sq / 2 + 8,
                    eps->stream));
  B.GH = eps->mred;
  B.M = B.GH + 2 * sq;
  B.theta_d = B.M + sq;
  B.res_d = B.theta_d + bp;
  double *bnd = B.res_d + bp, *gwork = bnd + 8;
  B.work = gwork + gw;
  B.work32 = reinterpret_cast<float *>(B.work + work_len);  // ctas * bp^2 floats
  B.err = reinterpret_cast<int *>(B.work32 + (size_t)ctas * sq);
  B.G.assign(sq, 0.0);
  B.H.assign(sq, 0.0);
  B.Q.assign(sq, 0.0);
  B.theta.assign(bp, 0.0);
  B.rel.assign(bp, 1.0);

  memset(&eps->stats, 0, sizeof(eps->stats));
  eps_monitor_start(eps);
  if (eps->timing) {
    cudaEventCreate(&B.f0);
    cudaEventCreate(&B.f1);
  }
  const uint64_t launches0 = launch_count();
  cudaEvent_t t0 = nullptr, t1 = nullptr, t2 = nullptr;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  cudaEventCreate(&t2);
  cudaEventRecord(t0, s);
  eps->nconv = 0;
  eps->its = 0;
  eps->reason = B200_CONVERGED_ITERATING;
  eps->solved = false;
  B200_CUDA_CHECK(cudaMemsetAsync(B.err, 0, sizeof(int), s));
  B200_CUDA_CHECK(mat_gershgorin(eps->A, bnd, gwork, gw, s));
  B200_CUDA_CHECK(cudaMemcpyAsync(B.bounds, bnd, sizeof(B.bounds), cudaMemcpyDeviceToHost, s));

  // start block: the initial space (EPSSetInitialSpace vectors, inserted into V by the setup), then
  // counter-based N(0,1) columns
  b200_bv_set_active_columns(V, 0, V->m);
  B200_CHECK(eps_insert_initial_space(eps, V, std::min(V->m, bp)));
  B.x32 = true;
  B.x = 0;
  B200_CUDA_CHECK(rb_init_launch(B.b32[0], true, n, bp, V->V, V->ld, eps->nini_eff, V->seed ^ 0x6d69786564ull, s));

  // ---------------------------------------------------------------- phase 1 (FP32 block)
  int sweeps1 = 0;
  B200_CHECK(B.svqb());
  B200_CHECK(B.rayleigh_ritz());
  double last = B.max_wanted();
  while (sweeps1 < max_sweeps && B.max_wanted() > tol_low) {
    const int d = B.choose_degree(tol_low, deg_cap);
    B.max_degree = std::max(B.max_degree, d);
    B200_CHECK(B.filter_segments(d, kSegCap32));
    B200_CHECK(B.svqb());
    B200_CHECK(B.rayleigh_ritz());
    B200_CHECK(B.monitor());
    ++sweeps1;
    const double now = B.max_wanted();
    if (now > 0.5 * last) break;  // no longer halving: the FP32 rounding floor
    last = now;
  }
  // The FP32 residual floor (about 1e-7: the block and A X are rounded to FP32) hides further
  // progress on the wanted pairs.  One more FP32 sweep, its degree taken from the Chebyshev growth
  // that brings the measured residuals to the FP64 target, converges the error components next to
  // the wanted end at half the bytes of an FP64 sweep; FP64 then only has to remove the broadband
  // rounding noise.
  if (tol < tol_low && sweeps1 < max_sweeps) {
    const int d = B.choose_degree(0.5 * tol, deg_cap);
    B.max_degree = std::max(B.max_degree, d);
    B200_CHECK(B.filter_segments(d, kSegCap32));
    B200_CHECK(B.svqb());
    B200_CHECK(B.rayleigh_ritz());
    B200_CHECK(B.monitor());
    ++sweeps1;
  }
  cudaEventRecord(t1, s);

  // ---------------------------------------------------------------- phase 2 (FP64 block)
  // The FP32 rounding noise of the block lies in every direction, so a short polish filter over a wide
  // interval (the unwanted spectrum up to kWide of the way from the block's weakest Ritz value) damps
  // it by kPolishGrowth in a few FP64 degrees; SVQB and the FP64 Rayleigh-Ritz step follow.
  B.x32 = false;
  B200_CUDA_CHECK(rb_widen_launch(B.b32[B.x], B.b64[0], (long long)blk, s));
  B.x = 0;
  int sweeps2 = 0;
  B200_CHECK(B.filter(B.polish_degree(kWide, kPolishGrowth, deg_cap), kWide));
  B200_CHECK(B.svqb());
  B200_CHECK(B.rayleigh_ritz());
  B200_CHECK(B.monitor());
  ++sweeps2;
  while (B.leading_converged(tol) < nev && sweeps2 < max_sweeps) {
    const int d = B.choose_degree(0.25 * tol, deg_cap);
    B.max_degree = std::max(B.max_degree, d);
    B200_CHECK(B.filter_segments(d, kSegCap64));
    B200_CHECK(B.svqb());
    B200_CHECK(B.rayleigh_ritz());
    B200_CHECK(B.monitor());
    ++sweeps2;
  }
  const int lead = B.leading_converged(tol);

  // results: the block's vectors in columns 0.. of the FP64 BV, values and residuals in wanted order
  const int ncopy = std::min(bp, V->m);
  B200_CUDA_CHECK(rb_to_colmajor_launch(B.b64[B.x], false, n, bp, ncopy, V->V, V->ld, s));
  for (int i = 0; i < (int)eps->perm.size(); ++i) eps->perm[i] = i;
  for (int i = 0; i < ncopy && i < (int)eps->eigr.size(); ++i) {
    eps->eigr[i] = B.theta[i];
    eps->errest[i] = B.rel[i];
  }
  eps->nconv = std::min(lead, ncopy);
  eps->its = sweeps1 + sweeps2;
  eps->reason = eps->nconv >= nev ? B200_CONVERGED_TOL : B200_DIVERGED_ITS;
  cudaEventRecord(t2, s);
  cudaEventSynchronize(t2);
  float ms1 = 0.f, ms2 = 0.f;
  cudaEventElapsedTime(&ms1, t0, t1);
  cudaEventElapsedTime(&ms2, t1, t2);
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  cudaEventDestroy(t2);
  eps->stats.phase1_restarts = sweeps1;  // FP32 sweeps
  eps->stats.filter_sweeps = sweeps2;    // FP64 sweeps
  eps->stats.filter_degree = B.max_degree;
  eps->stats.block_size = bp;
  eps->stats.spmm_columns = B.spmm_cols;
  eps->stats.ms_phase1 = ms1;
  eps->stats.ms_phase2 = ms2;
  eps->stats.ms_total = ms1 + ms2;
  eps->stats.kernel_launches = (int64_t)(launch_count() - launches0);
  eps->stats.ms_spmv = B.filter_ms;                // timing mode: the filters' block SpMVs
  eps->stats.gs_bytes = (int64_t)B.filter_bytes;   // and their algorithmic bytes
  eps->stats.gs_passes = B.svqb_count;             // block orthonormalisations (SVQB)
  eps->stats.ms_orth = B.svqb_ms;                  // timing mode: their wall time
  eps->stats.restarts = B.rr_count;                // Rayleigh-Ritz steps
  eps->stats.ms_restart = B.rr_ms;                 // timing mode: their wall time
  if (B.f0) cudaEventDestroy(B.f0);
  if (B.f1) cudaEventDestroy(B.f1);
  eps->solved = true;
  return B200_OK;
}
