// Batched Krylov-Schur: thousands of independent small Hermitian eigenproblems
// in one persistent launch.
//
// Every CTA takes problems from an atomic work queue (largest first) and runs
// the whole of EPSSolve_KrylovSchur_Default for one problem on its own
// (src/eps/impls/krylov/krylovschur/krylovschur.c:227-348, with the same
// decisions as the single-problem driver in lib.cu): Lanczos steps with the
// CSR SpMV in warp tiles (rows summed in index order), classical
// Gram-Schmidt with DGKS refinement "if needed" (bvorthog.c:91-217,
// eta 0.7071, at most three passes, the Pythagorean norm estimate), the
// projected problem on one warp (arrowhead to tridiagonal with Givens
// rotations as DSArrowTridiag, dshep.c:221-265; the symmetric tridiagonal
// eigenproblem by implicit QL iterations with Wilkinson shifts in place of
// LAPACK dsteqr; insertion sort, extra row and truncation as
// dshep.c:323-381,643-671), the convergence test of EPSKrylovConvergence with
// relative error estimates (epskrylov.c:207-295), the restart V = V Q in
// place and the final sort of SlepcSortEigenvalues.  No host round trip and
// no wait on another CTA: problems are independent.
//
// Determinism: every reduction is a fixed tree (per-thread row order, fixed
// shuffle tree, warps summed in order), the QL and sort run redundantly on
// the lanes of one warp (each lane owns one row of Q), so a batch gives the
// same bits run to run.  The basis is written and re-read by the same CTA
// between barriers; its loads go through L2 (ld.global.cg) so that they
// always see the CTA's own stores.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "common.h"
#include "internal.h"
#include "kernels.h"
#include "objects.h"

using namespace b200;

namespace b200 {
namespace {

constexpr int kBLd = 32;          // projected problem: ncv + 1 <= 32 (one warp owns its rows)
constexpr int kBCols = kBLd;      // basis columns incl. the Lanczos work column
constexpr double kBEps = 2.220446049250313e-16;

struct BProblem {
  long long rp_off;    // start of the problem's row pointer (n+1 local offsets)
  long long nnz_off;   // start of its nonzeros
  long long v_off;     // start of its basis: ld x (ncv + 1) doubles
  long long tile_off;  // first warp tile ({r0, r1, p0, p1} in local rows and nonzeros)
  long long x_off;     // start of its rows in the start-vector / output arrays
  long long nnz;       // its nonzeros
  int n, ld, ntiles, index;
};

struct BParams {
  int nev, ncv, mpd, max_it_user, which, pad;
  double tol, eta, keep;
  unsigned long long seed;
};

template <int T>
struct BShared {
  double red[T / 32][kBCols + 8];
  double c[kBCols + 8];
  double scal[8];    // scalars decided by thread 0 and read by every thread
  int flag[8];
  double d[kBLd], e[kBLd], Q[kBLd * kBLd], eigr[kBLd], errest[kBLd], wr[kBLd];
  double prod[T / 32][kWarpTileNnz];
  int perm[kBLd];
  int problem;
  unsigned long long bytes;  // algorithmic bytes moved for the current problem
};

__device__ __forceinline__ double bwarp_sum(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

__device__ __forceinline__ uint64_t bsplitmix(uint64_t z) {
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

// y = A x for one problem: warps walk its tiles (<= 32 rows, <= kWarpTileNnz nonzeros)
template <int T, typename XT>
__device__ void cta_spmv(const BProblem &P, const int *__restrict__ rowptr, const int *__restrict__ colind,
                         const double *__restrict__ vals, const int4 *__restrict__ tiles, const XT *x, double *y,
                         BShared<T> &sh) {
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  double *prod = sh.prod[wib];
  const int *rp = rowptr + P.rp_off;
  const int *ci = colind + P.nnz_off;
  const double *va = vals + P.nnz_off;
  for (int t = wib; t < P.ntiles; t += T / 32) {
    const int4 tile = tiles[P.tile_off + t];
    const int r0 = tile.x, r1 = tile.y, nrows = r1 - r0, p0 = tile.z, p1 = tile.w;
    const int mystart = (lane < nrows) ? rp[r0 + lane] : 0;
    const int nxt = __shfl_down_sync(0xffffffffu, mystart, 1);
    const int myend = (lane + 1 < nrows) ? nxt : p1;
    const int cnt = p1 - p0;
    for (int q = lane; q < cnt; q += 32) prod[q] = __dmul_rn(va[p0 + q], (double)__ldcg(x + ci[p0 + q]));
    __syncwarp();
    if (lane < nrows) {
      double s = 0.0;
      for (int q = mystart - p0; q < myend - p0; ++q) s = __dadd_rn(s, prod[q]);
      y[r0 + lane] = s;
    }
    __syncwarp();
  }
  __syncthreads();
}

// sh.c[i] = V(:,c0+i)' w for i < ncols (deterministic); w may be one of the columns.  Columns
// go in groups of 8: per-thread partial sums in row order, a fixed shuffle tree per warp, the
// warps added in order.
template <int T>
__device__ void cta_dots(const double *V, int ld, int n, int c0, int ncols, const double *w, BShared<T> &sh) {
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  if (threadIdx.x == 0) sh.bytes += 8ull * n * (ncols + 1);
  for (int g0 = 0; g0 < ncols; g0 += 8) {
    const int gn = min(8, ncols - g0);
    double acc[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) acc[i] = 0.0;
    for (int r = threadIdx.x; r < n; r += T) {
      const double wr = __ldcg(w + r);
#pragma unroll
      for (int i = 0; i < 8; ++i)
        if (i < gn) acc[i] = fma(__ldcg(V + r + (size_t)(c0 + g0 + i) * ld), wr, acc[i]);
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const double v = bwarp_sum(acc[i]);
      if (lane == 0) sh.red[wib][g0 + i] = v;
    }
  }
  __syncthreads();
  if (threadIdx.x < ncols) {
    double sacc = 0.0;
    for (int w2 = 0; w2 < T / 32; ++w2) sacc += sh.red[w2][threadIdx.x];
    sh.c[threadIdx.x] = sacc;
  }
  __syncthreads();
}

// w -= V(:,0:ncols) coef
template <int T>
__device__ void cta_update(const double *V, int ld, int n, int ncols, const double *coef, double *w) {
  for (int r = threadIdx.x; r < n; r += T) {
    double acc = 0.0;
    for (int i = 0; i < ncols; ++i) acc = fma(__ldcg(V + r + (size_t)i * ld), coef[i], acc);
    w[r] = __ldcg(w + r) - acc;
  }
  __syncthreads();
}

template <int T>
__device__ void cta_scale(double *w, int n, double alpha) {
  for (int r = threadIdx.x; r < n; r += T) w[r] = __ldcg(w + r) * alpha;
  __syncthreads();
}

template <int T>
__device__ void cta_copy(double *dst, const double *src, int n) {
  for (int r = threadIdx.x; r < n; r += T) dst[r] = __ldcg(src + r);
  __syncthreads();
}

// the random column of BVSetRandomColumn's stand-in (same generator as random_kernel)
template <int T>
__device__ void cta_random(double *w, int n, uint64_t seed, uint64_t stream_id) {
  for (int r = threadIdx.x; r < n; r += T) {
    const uint64_t z = bsplitmix(seed ^ bsplitmix(stream_id * 0x100000001B3ULL + (uint64_t)r));
    w[r] = (double)(z >> 11) * (1.0 / 9007199254740992.0);
  }
  __syncthreads();
}

// CGS + DGKS "if needed" of column j against columns 0..j-1 (bvorthog.c:91-217); on return
// h[0..j-1] holds the coefficients, *norm the norm of the new column, *lindep the flag.
// The column is then scaled by 1/norm unless the norm is 0 or 1 (BVOrthonormalizeColumn).
template <int T>
__device__ void cta_orthonormalize(double *V, int ld, int n, int j, double eta, double *h, double *norm, int *lindep,
                                   int *err, BShared<T> &sh) {
  double *w = V + (size_t)j * ld;
  for (int i = 0; i < j; ++i) h[i] = 0.0;
  int more = 1, passes = 0;
  while (more) {
    cta_dots<T>(V, ld, n, 0, j + 1, w, sh);  // includes w against itself
    for (int i = 0; i < j; ++i) h[i] += sh.c[i];
    cta_update<T>(V, ld, n, j, sh.c, w);
    if (threadIdx.x == 0 && j > 0) sh.bytes += 8ull * n * (j + 2);
    // thread 0: the Pythagorean estimate of the new norm (bvorthog.c:124-127)
    if (threadIdx.x == 0) {
      const double self = sh.c[j];
      if (self < 0.0) sh.flag[2] = 1;
      const double onrm = sqrt(self < 0.0 ? 0.0 : self);
      double sum = 0.0;
      for (int i = 0; i < j; ++i) sum += sh.c[i] * sh.c[i];
      const double est = onrm * onrm - sum;
      sh.scal[0] = onrm;
      sh.scal[1] = est;
      sh.flag[0] = est <= 0.0;
    }
    __syncthreads();
    double nrm;
    if (sh.flag[0]) {
      cta_dots<T>(V, ld, n, j, 1, w, sh);  // explicit norm
      nrm = sqrt(sh.c[0]);
    } else {
      nrm = sqrt(sh.scal[1]);
    }
    ++passes;
    if (threadIdx.x == 0) {
      const double onrm = sh.scal[0];
      sh.scal[2] = nrm;
      sh.flag[1] = (passes < 3 && nrm != 0.0 && fabs(nrm) < eta * fabs(onrm));
      sh.flag[3] = !(nrm != 0.0 && fabs(nrm) >= eta * fabs(onrm));
    }
    __syncthreads();
    more = sh.flag[1];
    __syncthreads();
  }
  const double nrm = sh.scal[2];
  *lindep = sh.flag[3];
  if (sh.flag[2]) *err = 1;
  *norm = nrm;
  __syncthreads();
  if (nrm != 1.0 && nrm != 0.0) {
    cta_scale<T>(w, n, 1.0 / nrm);
    if (threadIdx.x == 0) sh.bytes += 16ull * n;
  }
}

// plane rotation [c s; -s c] [f; g] = [r; 0] with r carrying the sign of f
__device__ __forceinline__ void givens(double f, double g, double *c, double *s, double *r) {
  if (g == 0.0) {
    *c = 1.0;
    *s = 0.0;
    *r = f;
  } else if (f == 0.0) {
    *c = 0.0;
    *s = (g > 0.0) ? 1.0 : -1.0;
    *r = fabs(g);
  } else {
    const double dd = hypot(f, g);
    *c = fabs(f) / dd;
    *r = copysign(dd, f);
    *s = g / *r;
  }
}

// The projected problem on warp 0: lanes own rows of Q (ld = kBLd); every lane computes the
// scalar recurrences, so all lanes hold the same d, e and permutation.
struct BDs {
  int n, l, k, t, state;  // state: 0 raw, 1 intermediate, 2 condensed, 3 truncated
};

__device__ void ds_solve(BDs &ds, double *d, double *e, double *Q, double *wr, int lane) {
  const int ld = kBLd, l = ds.l, n = ds.n;
  // DSSetIdentity on columns l..n-1
  for (int c = l; c < n; ++c) Q[lane + c * ld] = (lane == c) ? 1.0 : 0.0;
  __syncwarp();
  if (ds.state < 1) {
    // DSArrowTridiag of the (k-l+1) arrowhead at offset l (dshep.c:221-265)
    int na = ds.k - l + 1;
    if (na < 0) na = 0;
    double *dd = d + l, *ee = e + l;
    for (int j = 0; j + 2 < na; ++j) {
      double c, s, r;
      givens(ee[j + 1], ee[j], &c, &s, &r);
      ee[j + 1] = r;
      s = -s;
      double temp = dd[j + 1];
      ee[j] = c * s * (temp - dd[j]);
      dd[j + 1] = s * s * dd[j] + c * c * temp;
      dd[j] = c * c * dd[j] + s * s * temp;
      if (lane < j + 2) {
        double *qa = Q + (l + j) * ld + l, *qb = Q + (l + j + 1) * ld + l;
        const double x = qa[lane], y = qb[lane];
        qa[lane] = c * x + s * y;
        qb[lane] = c * y - s * x;
      }
      for (int i = j - 1; i >= 0; --i) {
        const double off = -s * ee[i];
        ee[i] = c * ee[i];
        temp = ee[i + 1];
        givens(temp, off, &c, &s, &r);
        ee[i + 1] = r;
        s = -s;
        temp = (dd[i] - dd[i + 1]) * s - 2.0 * c * ee[i];
        const double p = s * temp;
        dd[i + 1] += p;
        dd[i] -= p;
        ee[i] = -ee[i] - c * temp;
        if (lane < j + 2) {
          double *qa = Q + (l + i) * ld + l, *qb = Q + (l + i + 1) * ld + l;
          const double x = qa[lane], y = qb[lane];
          qa[lane] = c * x + s * y;
          qb[lane] = c * y - s * x;
        }
      }
    }
    __syncwarp();
  }
  for (int i = 0; i < l; ++i) wr[i] = d[i];
  // symmetric tridiagonal eigenproblem of d[l..n), e[l..n-1) by implicit QL with Wilkinson shifts,
  // rotations accumulated into columns l..n-1 of Q
  const int m0 = n - l;
  double *dd = d + l, *ee = e + l;
  const double extra = (n > 0) ? e[n - 1] : 0.0;  // the Lanczos beta kept for DSUpdateExtraRow
  if (m0 > 0) ee[m0 - 1] = 0.0;
  for (int L = 0; L < m0; ++L) {
    for (int iter = 0; iter < 60 * kBLd; ++iter) {
      int m = L;
      for (; m < m0 - 1; ++m) {
        const double dsum = fabs(dd[m]) + fabs(dd[m + 1]);
        if (fabs(ee[m]) <= kBEps * dsum) break;
      }
      if (m == L) break;
      double g = (dd[L + 1] - dd[L]) / (2.0 * ee[L]);
      double r = hypot(g, 1.0);
      g = dd[m] - dd[L] + ee[L] / (g + copysign(r, g));
      double s = 1.0, c = 1.0, p = 0.0;
      int i = m - 1;
      bool deflated = false;
      for (; i >= L; --i) {
        double f = s * ee[i];
        const double b = c * ee[i];
        r = hypot(f, g);
        ee[i + 1] = r;
        if (r == 0.0) {
          dd[i + 1] -= p;
          ee[m] = 0.0;
          deflated = true;
          break;
        }
        s = f / r;
        c = g / r;
        g = dd[i + 1] - p;
        r = (dd[i] - g) * s + 2.0 * c * b;
        p = s * r;
        dd[i + 1] = g + p;
        g = c * r - b;
        // rotate columns l+i and l+i+1 of Q
        double *qa = Q + (l + i) * ld, *qb = Q + (l + i + 1) * ld;
        f = qb[lane];
        qb[lane] = s * qa[lane] + c * f;
        qa[lane] = c * qa[lane] - s * f;
      }
      __syncwarp();
      if (deflated && i >= L) continue;
      dd[L] -= p;
      ee[L] = g;
      ee[m] = 0.0;
    }
  }
  for (int i = l; i < n; ++i) wr[i] = d[i];
  for (int i = 0; i < n - 1; ++i) e[i] = 0.0;
  if (n > 0) e[n - 1] = extra;
  ds.state = 2;
  __syncwarp();
}

__device__ __forceinline__ int bcompare(int which, double a, double b) {
  switch (which) {
    case B200_LARGEST_MAGNITUDE: {
      const double x = fabs(a), y = fabs(b);
      return (x < y) ? 1 : (x > y) ? -1 : 0;
    }
    case B200_SMALLEST_MAGNITUDE: {
      const double x = fabs(a), y = fabs(b);
      return (x > y) ? 1 : (x < y) ? -1 : 0;
    }
    case B200_LARGEST_REAL:
      return (a < b) ? 1 : (a > b) ? -1 : 0;
    default:
      return (a > b) ? 1 : (a < b) ? -1 : 0;
  }
}

// DSSort_HEP: insertion sort of d[l..t) then the column permutation of Q (row per lane)
__device__ void ds_sort(BDs &ds, double *d, double *Q, double *wr, int *perm, int which, int lane) {
  const int l = ds.l, n = ds.n, ld = kBLd;
  int pm[kBLd];
  for (int i = 0; i < n; ++i) pm[i] = i;
  for (int i = l + 1; i < ds.t; ++i) {
    const double re = d[pm[i]];
    int j = i - 1;
    int result = bcompare(which, re, d[pm[j]]);
    while (result < 0 && j >= l) {
      const int tmp = pm[j];
      pm[j] = pm[j + 1];
      pm[j + 1] = tmp;
      --j;
      if (j >= l) result = bcompare(which, re, d[pm[j]]);
    }
  }
  double w2[kBLd];
  for (int i = l; i < n; ++i) w2[i] = d[pm[i]];
  for (int i = l; i < n; ++i) wr[i] = w2[i];
  for (int i = l; i < n; ++i) {
    const int p = pm[i];
    if (p != i) {
      int j = i + 1;
      while (pm[j] != i) ++j;
      pm[j] = p;
      pm[i] = i;
      const double tmp = Q[lane + p * ld];
      Q[lane + p * ld] = Q[lane + i * ld];
      Q[lane + i * ld] = tmp;
    }
  }
  for (int i = l; i < n; ++i) d[i] = wr[i];
  if (lane == 0)
    for (int i = 0; i < n; ++i) perm[i] = pm[i];
  __syncwarp();
}

// V(:, s:e) = V(:, l:k) Q(l:k, s:e) in place, row by row (each thread reads its rows before writing)
template <int T>
__device__ void cta_multinplace(double *V, int ld, int n, int l, int k, const double *Q, int s, int e) {
  if (e <= s || k <= l) return;
  for (int r = threadIdx.x; r < n; r += T) {
    double row[kBCols];
#pragma unroll
    for (int c = 0; c < kBCols; ++c)
      if (c < k - l) row[c] = __ldcg(V + r + (size_t)(l + c) * ld);
    for (int j = s; j < e; ++j) {
      double acc = 0.0;
#pragma unroll
      for (int c = 0; c < kBCols; ++c)
        if (c < k - l) acc = fma(row[c], Q[(l + c) + j * kBLd], acc);
      V[r + (size_t)j * ld] = acc;
    }
  }
  __syncthreads();
}

template <int T>
__global__ void __launch_bounds__(T) batched_ks_kernel(int nprob, const BProblem *__restrict__ probs,
                                                       const int *__restrict__ order, int *__restrict__ next,
                                                       const int *__restrict__ rowptr, const int *__restrict__ colind,
                                                       const double *__restrict__ vals, const int4 *__restrict__ tiles,
                                                       const double *__restrict__ v0, double *Vall,
                                                       BParams prm, double *__restrict__ evals,
                                                       double *__restrict__ errest_out, int *__restrict__ vcol,
                                                       int *__restrict__ info, double *__restrict__ bytes_out) {
  __shared__ BShared<T> sh;
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  for (;;) {
    if (threadIdx.x == 0) {
      const int q = atomicAdd(next, 1);
      sh.problem = q < nprob ? order[q] : -1;
    }
    __syncthreads();
    const int pidx = sh.problem;
    __syncthreads();
    if (pidx < 0) return;
    const BProblem P = probs[pidx];
    const int n = P.n, ld = P.ld;
    double *V = Vall + P.v_off;
    const int ncv = prm.ncv, mpd = prm.mpd, nev = prm.nev;
    const int max_it = prm.max_it_user > 0 ? prm.max_it_user : max(100, 2 * n / ncv);
    int err = 0;
    uint64_t nrand = 0;
    if (threadIdx.x < 8) sh.flag[threadIdx.x] = 0;
    if (threadIdx.x == 0) sh.bytes = 0;
    __syncthreads();
    BDs ds{0, 0, 0, 0, 0};
    double h[kBCols + 1];
    // EPSSetUp: BVInsertVecs of the start vector (dropped if zero), then EPSGetStartVector(0)
    int nini = 0;
    {
      cta_copy<T>(V, v0 + P.x_off, n);
      double nrm;
      int lindep;
      cta_orthonormalize<T>(V, ld, n, 0, prm.eta, h, &nrm, &lindep, &err, sh);
      nini = (nrm == 0.0 || lindep) ? 0 : 1;
      if (!nini) cta_random<T>(V, n, prm.seed, nrand++);
      cta_orthonormalize<T>(V, ld, n, 0, prm.eta, h, &nrm, &lindep, &err, sh);
      if (nrm == 0.0 || lindep) err = 2;
    }
    int nconv = 0, its = 0, reason = 0, l = 0;
    long long steps = 0;
    double beta = 0.0;
    if (threadIdx.x < kBLd) {
      sh.d[threadIdx.x] = 0.0;
      sh.e[threadIdx.x] = 0.0;
    }
    __syncthreads();
    while (reason == 0 && !err) {
      ++its;
      int nv = min(nconv + mpd, ncv);
      ds.n = nv;
      ds.t = nv;
      ds.l = nconv;
      ds.k = nconv + l;
      // BVMatLanczos from column k
      const int k0 = nconv + l;
      int m = nv, breakdown = 0;
      for (int j = k0; j < m; ++j) {
        cta_spmv<T, double>(P, rowptr, colind, vals, tiles, V + (size_t)j * ld, V + (size_t)(j + 1) * ld, sh);
        if (threadIdx.x == 0) sh.bytes += 12ull * P.nnz + 4ull * (n + 1) + 16ull * n;
        double nrm;
        int lindep;
        cta_orthonormalize<T>(V, ld, n, j + 1, prm.eta, h, &nrm, &lindep, &err, sh);
        if (threadIdx.x == 0) {
          sh.d[j] = h[j];
          sh.e[j] = lindep ? 0.0 : nrm;  // BV_SetValue stores 0 for a dependent column
        }
        ++steps;
        beta = nrm;
        if (lindep) {
          m = j + 1;
          breakdown = 1;
          break;
        }
      }
      __syncthreads();
      nv = m;
      ds.n = nv;
      ds.t = nv;
      ds.l = nconv;
      ds.k = nconv + l;
      ds.state = l ? 0 : 1;
      if (wib == 0) {
        ds_solve(ds, sh.d, sh.e, sh.Q, sh.wr, lane);
        ds_sort(ds, sh.d, sh.Q, sh.wr, sh.perm, prm.which, lane);
        // DSUpdateExtraRow_HEP
        const double bt = sh.e[ds.n - 1];
        __syncwarp();
        if (lane < ds.n) sh.e[lane] = bt * sh.Q[ds.n - 1 + lane * kBLd];
        __syncwarp();
      }
      ds.k = ds.n;
      ds.state = 2;
      __syncthreads();
      // EPSKrylovConvergence with the relative test
      int kk = nconv;
      for (; kk < nv; ++kk) {
        const double re = sh.wr[kk];
        const double resnorm = fabs(sh.Q[ds.n - 1 + kk * kBLd]) * beta;
        const double wabs = fabs(re);
        const double est = (wabs != 0.0) ? resnorm / wabs : 1.7976931348623157e308;
        if (threadIdx.x == 0) {
          sh.eigr[kk] = re;
          sh.errest[kk] = est;
        }
        if (est >= prm.tol) break;
      }
      const int k = kk;
      if (k >= nev) reason = B200_CONVERGED_TOL;
      else if (its >= max_it) reason = B200_DIVERGED_ITS;
      int lnew;
      if (reason != 0 || breakdown || k == nv) lnew = 0;
      else {
        lnew = (int)((nv - k) * prm.keep);
        if (lnew < 1) lnew = 1;
      }
      __syncthreads();
      if (reason == 0) {
        if (breakdown || k == nv) {
          if (k < nev) {
            // EPSGetStartVector(eps,k,&breakdown): a random column orthonormalised against 0..k-1
            cta_random<T>(V + (size_t)k * ld, n, prm.seed, nrand++);
            double nrm;
            int lindep;
            cta_orthonormalize<T>(V, ld, n, k, prm.eta, h, &nrm, &lindep, &err, sh);
            if (lindep) reason = B200_DIVERGED_BREAKDOWN;
          }
        } else {
          // DSTruncate_HEP(k + lnew)
          ds.k = k + lnew;
          ds.t = ds.n;
          ds.n = k + lnew;
          ds.state = 3;
        }
      }
      // BVMultInPlace(V, Q, nconv, k + lnew) on the active columns [nconv, nv)
      {
        const int s = nconv, e = k + lnew;
        if (e > s) {
          // Q restricted to rows [nconv, nv): V(:, s:e) = V(:, nconv:nv) Q(nconv:nv, s:e)
          cta_multinplace<T>(V, ld, n, nconv, nv, sh.Q, s, e);
          if (threadIdx.x == 0) sh.bytes += 8ull * n * ((nv - nconv) + (e - s));
        }
      }
      if (reason == 0 && !breakdown) cta_copy<T>(V + (size_t)(k + lnew) * ld, V + (size_t)nv * ld, n);
      nconv = k;
      l = lnew;
      __syncthreads();
    }
    // SlepcSortEigenvalues and outputs
    if (threadIdx.x == 0) {
      int pm[kBLd];
      for (int i = 0; i < ncv; ++i) pm[i] = i;
      for (int i = nconv - 1; i >= 0; --i) {
        const double re = sh.eigr[pm[i]];
        int j = i + 1;
        while (j < nconv) {
          if (bcompare(prm.which, re, sh.eigr[pm[j]]) <= 0) break;
          const int tmp = pm[j - 1];
          pm[j - 1] = pm[j];
          pm[j] = tmp;
          ++j;
        }
      }
      for (int i = 0; i < ncv; ++i) {
        evals[(size_t)pidx * ncv + i] = i < nconv ? sh.eigr[pm[i]] : 0.0;
        errest_out[(size_t)pidx * ncv + i] = i < nconv ? sh.errest[pm[i]] : 0.0;
        vcol[(size_t)pidx * ncv + i] = i < nconv ? pm[i] : -1;
      }
      int *inf = info + (size_t)pidx * 8;
      inf[0] = nconv;
      inf[1] = its;
      inf[2] = reason;
      inf[3] = (int)steps;
      inf[4] = err;
      inf[5] = nini;
      bytes_out[pidx] = (double)sh.bytes;
    }
    __syncthreads();
  }
}

// ---- FP32 basis (phase 1 of the mixed form): the basis columns are stored as FP32, the vector
// being orthogonalised is a separate FP64 work vector, every product and sum is FP64.

// sh.c[i] = V32(:,i)' w for i < ncols and sh.c[ncols] = w' w (deterministic, groups of 8 columns)
template <int T>
__device__ void cta_dots32(const float *V, int ld, int n, int ncols, const double *w, BShared<T> &sh) {
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  if (threadIdx.x == 0) sh.bytes += 4ull * n * ncols + 8ull * n;
  for (int g0 = 0; g0 < ncols || g0 == 0; g0 += 8) {
    const int gn = min(8, ncols - g0);
    double acc[8], self = 0.0;
#pragma unroll
    for (int i = 0; i < 8; ++i) acc[i] = 0.0;
    for (int r = threadIdx.x; r < n; r += T) {
      const double wr = __ldcg(w + r);
#pragma unroll
      for (int i = 0; i < 8; ++i)
        if (i < gn) acc[i] = fma((double)__ldcg(V + r + (size_t)(g0 + i) * ld), wr, acc[i]);
      if (g0 == 0) self = fma(wr, wr, self);
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const double v = bwarp_sum(acc[i]);
      if (lane == 0 && i < gn) sh.red[wib][g0 + i] = v;
    }
    if (g0 == 0) {
      const double v = bwarp_sum(self);
      if (lane == 0) sh.red[wib][ncols] = v;
    }
  }
  __syncthreads();
  if (threadIdx.x <= ncols) {
    double sacc = 0.0;
    for (int w2 = 0; w2 < T / 32; ++w2) sacc += sh.red[w2][threadIdx.x];
    sh.c[threadIdx.x] = sacc;
  }
  __syncthreads();
}

// w -= V32(:,0:ncols) coef
template <int T>
__device__ void cta_update32(const float *V, int ld, int n, int ncols, const double *coef, double *w) {
  for (int r = threadIdx.x; r < n; r += T) {
    double acc = 0.0;
    for (int i = 0; i < ncols; ++i) acc = fma((double)__ldcg(V + r + (size_t)i * ld), coef[i], acc);
    w[r] = __ldcg(w + r) - acc;
  }
  __syncthreads();
}

// CGS + DGKS "if needed" of the FP64 vector w against the FP32 columns 0..j-1 (the same decisions
// as cta_orthonormalize), w scaled by 1/norm, then rounded into column j of the basis.
template <int T>
__device__ void cta_orth32(float *V, int ld, int n, int j, double *w, double eta, double *h, double *norm,
                           int *lindep, int *err, BShared<T> &sh) {
  for (int i = 0; i < j; ++i) h[i] = 0.0;
  int more = 1, passes = 0;
  while (more) {
    cta_dots32<T>(V, ld, n, j, w, sh);
    for (int i = 0; i < j; ++i) h[i] += sh.c[i];
    cta_update32<T>(V, ld, n, j, sh.c, w);
    if (threadIdx.x == 0 && j > 0) sh.bytes += 4ull * n * j + 16ull * n;
    if (threadIdx.x == 0) {
      const double self = sh.c[j];
      if (self < 0.0) sh.flag[2] = 1;
      const double onrm = sqrt(self < 0.0 ? 0.0 : self);
      double sum = 0.0;
      for (int i = 0; i < j; ++i) sum += sh.c[i] * sh.c[i];
      const double est = onrm * onrm - sum;
      sh.scal[0] = onrm;
      sh.scal[1] = est;
      sh.flag[0] = est <= 0.0;
    }
    __syncthreads();
    double nrm;
    if (sh.flag[0]) {
      cta_dots32<T>(V, ld, n, 0, w, sh);  // explicit norm
      nrm = sqrt(sh.c[0]);
    } else {
      nrm = sqrt(sh.scal[1]);
    }
    ++passes;
    if (threadIdx.x == 0) {
      const double onrm = sh.scal[0];
      sh.scal[2] = nrm;
      sh.flag[1] = (passes < 3 && nrm != 0.0 && fabs(nrm) < eta * fabs(onrm));
      sh.flag[3] = !(nrm != 0.0 && fabs(nrm) >= eta * fabs(onrm));
    }
    __syncthreads();
    more = sh.flag[1];
    __syncthreads();
  }
  const double nrm = sh.scal[2];
  *lindep = sh.flag[3];
  if (sh.flag[2]) *err = 1;
  *norm = nrm;
  __syncthreads();
  const double sc = (nrm != 1.0 && nrm != 0.0) ? 1.0 / nrm : 1.0;
  float *col = V + (size_t)j * ld;
  for (int r = threadIdx.x; r < n; r += T) {
    const double v = __ldcg(w + r) * sc;
    w[r] = v;
    col[r] = __double2float_rn(v);
  }
  if (threadIdx.x == 0) sh.bytes += 20ull * n;
  __syncthreads();
}

// V32(:, s:e) = V32(:, l:k) Q(l:k, s:e) in place (FP64 sums)
template <int T>
__device__ void cta_multinplace32(float *V, int ld, int n, int l, int k, const double *Q, int s, int e) {
  if (e <= s || k <= l) return;
  for (int r = threadIdx.x; r < n; r += T) {
    double row[kBCols];
#pragma unroll
    for (int c = 0; c < kBCols; ++c)
      if (c < k - l) row[c] = (double)__ldcg(V + r + (size_t)(l + c) * ld);
    for (int j = s; j < e; ++j) {
      double acc = 0.0;
#pragma unroll
      for (int c = 0; c < kBCols; ++c)
        if (c < k - l) acc = fma(row[c], Q[(l + c) + j * kBLd], acc);
      V[r + (size_t)j * ld] = __double2float_rn(acc);
    }
  }
  __syncthreads();
}

// Phase 1 of the batched mixed form: batched_ks_kernel's loop on an FP32 basis (same decisions,
// same projected-problem code), stopping at prm.tol (the loose tolerance).  W holds one FP64 work
// vector per problem (at the problem's row offset).
template <int T>
__global__ void __launch_bounds__(T) batched_ks32_kernel(int nprob, const BProblem *__restrict__ probs,
                                                         const int *__restrict__ order, int *__restrict__ next,
                                                         const int *__restrict__ rowptr,
                                                         const int *__restrict__ colind,
                                                         const double *__restrict__ vals,
                                                         const int4 *__restrict__ tiles,
                                                         const double *__restrict__ v0, float *Vall, double *Wall,
                                                         BParams prm, double *__restrict__ evals,
                                                         double *__restrict__ errest_out, int *__restrict__ vcol,
                                                         int *__restrict__ info, double *__restrict__ bytes_out) {
  __shared__ BShared<T> sh;
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  for (;;) {
    if (threadIdx.x == 0) {
      const int q = atomicAdd(next, 1);
      sh.problem = q < nprob ? order[q] : -1;
    }
    __syncthreads();
    const int pidx = sh.problem;
    __syncthreads();
    if (pidx < 0) return;
    const BProblem P = probs[pidx];
    const int n = P.n, ld = P.ld;
    float *V = Vall + P.v_off;
    double *w = Wall + P.x_off;
    const int ncv = prm.ncv, mpd = prm.mpd, nev = prm.nev;
    const int max_it = prm.max_it_user > 0 ? prm.max_it_user : max(100, 2 * n / ncv);
    int err = 0;
    uint64_t nrand = 0;
    if (threadIdx.x < 8) sh.flag[threadIdx.x] = 0;
    if (threadIdx.x == 0) sh.bytes = 0;
    __syncthreads();
    BDs ds{0, 0, 0, 0, 0};
    double h[kBCols + 1];
    int nini = 0;
    {
      cta_copy<T>(w, v0 + P.x_off, n);
      double nrm;
      int lindep;
      cta_orth32<T>(V, ld, n, 0, w, prm.eta, h, &nrm, &lindep, &err, sh);
      nini = (nrm == 0.0 || lindep) ? 0 : 1;
      if (!nini) {
        cta_random<T>(w, n, prm.seed, nrand++);
        cta_orth32<T>(V, ld, n, 0, w, prm.eta, h, &nrm, &lindep, &err, sh);
      }
      if (nrm == 0.0 || lindep) err = 2;
    }
    int nconv = 0, its = 0, reason = 0, l = 0;
    long long steps = 0;
    double beta = 0.0;
    if (threadIdx.x < kBLd) {
      sh.d[threadIdx.x] = 0.0;
      sh.e[threadIdx.x] = 0.0;
    }
    __syncthreads();
    while (reason == 0 && !err) {
      ++its;
      int nv = min(nconv + mpd, ncv);
      ds.n = nv;
      ds.t = nv;
      ds.l = nconv;
      ds.k = nconv + l;
      const int k0 = nconv + l;
      int m = nv, breakdown = 0;
      for (int j = k0; j < m; ++j) {
        cta_spmv<T, float>(P, rowptr, colind, vals, tiles, V + (size_t)j * ld, w, sh);
        if (threadIdx.x == 0) sh.bytes += 12ull * P.nnz + 4ull * (n + 1) + 12ull * n;
        double nrm;
        int lindep;
        cta_orth32<T>(V, ld, n, j + 1, w, prm.eta, h, &nrm, &lindep, &err, sh);
        if (threadIdx.x == 0) {
          sh.d[j] = h[j];
          sh.e[j] = lindep ? 0.0 : nrm;
        }
        ++steps;
        beta = nrm;
        if (lindep) {
          m = j + 1;
          breakdown = 1;
          break;
        }
      }
      __syncthreads();
      nv = m;
      ds.n = nv;
      ds.t = nv;
      ds.l = nconv;
      ds.k = nconv + l;
      ds.state = l ? 0 : 1;
      if (wib == 0) {
        ds_solve(ds, sh.d, sh.e, sh.Q, sh.wr, lane);
        ds_sort(ds, sh.d, sh.Q, sh.wr, sh.perm, prm.which, lane);
        const double bt = sh.e[ds.n - 1];
        __syncwarp();
        if (lane < ds.n) sh.e[lane] = bt * sh.Q[ds.n - 1 + lane * kBLd];
        __syncwarp();
      }
      ds.k = ds.n;
      ds.state = 2;
      __syncthreads();
      int kk = nconv;
      for (; kk < nv; ++kk) {
        const double re = sh.wr[kk];
        const double resnorm = fabs(sh.Q[ds.n - 1 + kk * kBLd]) * beta;
        const double wabs = fabs(re);
        const double est = (wabs != 0.0) ? resnorm / wabs : 1.7976931348623157e308;
        if (threadIdx.x == 0) {
          sh.eigr[kk] = re;
          sh.errest[kk] = est;
        }
        if (est >= prm.tol) break;
      }
      const int k = kk;
      if (k >= nev) reason = B200_CONVERGED_TOL;
      else if (its >= max_it) reason = B200_DIVERGED_ITS;
      int lnew;
      if (reason != 0 || breakdown || k == nv) lnew = 0;
      else {
        lnew = (int)((nv - k) * prm.keep);
        if (lnew < 1) lnew = 1;
      }
      __syncthreads();
      if (reason == 0) {
        if (breakdown || k == nv) {
          if (k < nev) {
            cta_random<T>(w, n, prm.seed, nrand++);
            double nrm;
            int lindep;
            cta_orth32<T>(V, ld, n, k, w, prm.eta, h, &nrm, &lindep, &err, sh);
            if (lindep) reason = B200_DIVERGED_BREAKDOWN;
          }
        } else {
          ds.k = k + lnew;
          ds.t = ds.n;
          ds.n = k + lnew;
          ds.state = 3;
        }
      }
      {
        const int s = nconv, e = k + lnew;
        if (e > s) {
          cta_multinplace32<T>(V, ld, n, nconv, nv, sh.Q, s, e);
          if (threadIdx.x == 0) sh.bytes += 4ull * n * ((nv - nconv) + (e - s));
        }
      }
      if (reason == 0 && !breakdown) {
        const float *src = V + (size_t)nv * ld;
        float *dst = V + (size_t)(k + lnew) * ld;
        for (int r = threadIdx.x; r < n; r += T) dst[r] = __ldcg(src + r);
        __syncthreads();
      }
      nconv = k;
      l = lnew;
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      int pm[kBLd];
      for (int i = 0; i < ncv; ++i) pm[i] = i;
      for (int i = nconv - 1; i >= 0; --i) {
        const double re = sh.eigr[pm[i]];
        int j = i + 1;
        while (j < nconv) {
          if (bcompare(prm.which, re, sh.eigr[pm[j]]) <= 0) break;
          const int tmp = pm[j - 1];
          pm[j - 1] = pm[j];
          pm[j] = tmp;
          ++j;
        }
      }
      for (int i = 0; i < ncv; ++i) {
        evals[(size_t)pidx * ncv + i] = i < nconv ? sh.eigr[pm[i]] : 0.0;
        errest_out[(size_t)pidx * ncv + i] = i < nconv ? sh.errest[pm[i]] : 0.0;
        vcol[(size_t)pidx * ncv + i] = i < nconv ? pm[i] : -1;
      }
      int *inf = info + (size_t)pidx * 8;
      inf[0] = nconv;
      inf[1] = its;
      inf[2] = reason;
      inf[3] = (int)steps;
      inf[4] = err;
      inf[5] = nini;
      bytes_out[pidx] = (double)sh.bytes;
    }
    __syncthreads();
  }
}

// The start vector of phase 2 for every problem: the sum of its (up to nev) phase-1 Ritz vectors
// in FP64, or its original start vector when phase 1 converged none; phase 1's counters are kept.
__global__ void batched_phase2_start_kernel(int nprob, const BProblem *__restrict__ probs, int nev, int ncv,
                                            const float *__restrict__ V32, const int *__restrict__ vcol,
                                            const int *__restrict__ info, const double *__restrict__ bytes,
                                            const double *__restrict__ v0, double *__restrict__ v0_next,
                                            int *__restrict__ info1, double *__restrict__ bytes1) {
  for (int p = blockIdx.x; p < nprob; p += gridDim.x) {
    const BProblem P = probs[p];
    const int nconv = min(info[(size_t)p * 8], nev);
    const float *V = V32 + P.v_off;
    for (int r = threadIdx.x; r < P.n; r += blockDim.x) {
      double s = 0.0;
      for (int i = 0; i < nconv; ++i) s += (double)V[r + (size_t)vcol[(size_t)p * ncv + i] * P.ld];
      v0_next[P.x_off + r] = nconv > 0 ? s : v0[P.x_off + r];
    }
    if (threadIdx.x < 8) info1[(size_t)p * 8 + threadIdx.x] = info[(size_t)p * 8 + threadIdx.x];
    if (threadIdx.x == 0) bytes1[p] = bytes[p];
  }
}

}  // namespace
}  // namespace b200

// ------------------------------------------------------------------ host side ---
struct b200_batch_s {
  cudaStream_t stream = nullptr;
  int nprob = 0;
  std::vector<int> ns;
  std::vector<b200::BProblem> hprobs;
  b200::BProblem *probs = nullptr;
  int *rowptr = nullptr, *colind = nullptr;
  double *vals = nullptr;
  int4 *tiles = nullptr;
  double *v0 = nullptr;   // concatenated start vectors
  double *V = nullptr;    // concatenated bases
  size_t v_total = 0;
  int *order = nullptr;   // problems by decreasing size
  int *next = nullptr;    // work-queue counter
  double *evals = nullptr, *errest = nullptr;
  int *vcol = nullptr, *info = nullptr;
  double *bytes = nullptr;  // algorithmic bytes per problem of the last solve
  long long total_rows = 0;
  // parameters
  int nev = 1, ncv = 0, mpd = 0, max_it = 0, which = B200_LARGEST_REAL;
  double tol = 1e-8;
  int threads = 0;        // 0: chosen by the autotuner on the first solve
  // results on the host
  std::vector<double> h_evals, h_errest;
  std::vector<int> h_vcol, h_info;
  std::vector<double> h_bytes;
  bool solved = false;
  // captured launch
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int graph_threads = 0;
  b200::BParams graph_prm{};
  int alloc_ncv = 0;
  float last_ms = 0.0f;
  // mixed precision: phase 1 on an FP32 basis to tol_low, phase 2 in FP64 from the phase-1 Ritz vectors
  int precision = B200_PRECISION_FP64;
  double tol_low = 1e-6;
  float *V32 = nullptr;      // FP32 bases (same offsets as V)
  double *W = nullptr;       // FP64 work vector per problem (row offsets)
  double *v0_2 = nullptr;    // phase-2 start vectors
  int *info1 = nullptr;      // phase-1 counters (nprob x 8)
  double *bytes1 = nullptr;  // phase-1 algorithmic bytes per problem
  std::vector<int> h_info1;
  std::vector<double> h_bytes1;
  int graph_precision = -1;
  double graph_tol_low = 0.0;
};

namespace b200 {
namespace {

template <int T>
cudaError_t launch_batched(b200_batch B, const b200::BParams &prm, int nprob, cudaStream_t s, bool count,
                           const double *v0 = nullptr) {
  int sms = num_sms_host(), per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batched_ks_kernel<T>, T, 0);
  if (per_sm < 1) per_sm = 1;
  int grid = sms * per_sm;
  if (grid > nprob) grid = nprob;
  cudaError_t e = cudaMemsetAsync(B->next, 0, sizeof(int), s);
  if (e != cudaSuccess) return e;
  // every info entry -1 until its problem is solved
  e = cudaMemsetAsync(B->info, 0xff, sizeof(int) * 8 * (size_t)B->nprob, s);
  if (e != cudaSuccess) return e;
  batched_ks_kernel<T><<<grid, T, 0, s>>>(nprob, B->probs, B->order, B->next, B->rowptr, B->colind, B->vals,
                                          B->tiles, v0 ? v0 : B->v0, B->V, prm, B->evals, B->errest, B->vcol,
                                          B->info, B->bytes);
  if (count) count_launch();
  return cudaGetLastError();
}

// The mixed form: phase 1 (FP32 basis, tolerance tol_low), the phase-2 start vectors, phase 2 (FP64).
template <int T>
cudaError_t launch_mixed(b200_batch B, const b200::BParams &prm, cudaStream_t s, bool count) {
  int sms = num_sms_host(), per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batched_ks32_kernel<T>, T, 0);
  if (per_sm < 1) per_sm = 1;
  int grid = sms * per_sm;
  if (grid > B->nprob) grid = B->nprob;
  cudaError_t e = cudaMemsetAsync(B->next, 0, sizeof(int), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(B->info, 0xff, sizeof(int) * 8 * (size_t)B->nprob, s);
  if (e != cudaSuccess) return e;
  b200::BParams p1 = prm;
  p1.tol = B->tol_low > prm.tol ? B->tol_low : prm.tol;
  batched_ks32_kernel<T><<<grid, T, 0, s>>>(B->nprob, B->probs, B->order, B->next, B->rowptr, B->colind, B->vals,
                                            B->tiles, B->v0, B->V32, B->W, p1, B->evals, B->errest, B->vcol,
                                            B->info, B->bytes);
  if (count) count_launch();
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  const int g2 = B->nprob < sms * 8 ? B->nprob : sms * 8;
  batched_phase2_start_kernel<<<g2, 256, 0, s>>>(B->nprob, B->probs, prm.nev, prm.ncv, B->V32, B->vcol, B->info,
                                                 B->bytes, B->v0, B->v0_2, B->info1, B->bytes1);
  if (count) count_launch();
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  return launch_batched<T>(B, prm, B->nprob, s, count, B->v0_2);
}

cudaError_t launch_mixed_any(b200_batch B, int threads, const b200::BParams &prm, cudaStream_t s, bool count) {
  switch (threads) {
    case 128: return launch_mixed<128>(B, prm, s, count);
    case 256: return launch_mixed<256>(B, prm, s, count);
    default: return launch_mixed<512>(B, prm, s, count);
  }
}

cudaError_t launch_any(b200_batch B, int threads, const b200::BParams &prm, int nprob, cudaStream_t s, bool count) {
  switch (threads) {
    case 128: return launch_batched<128>(B, prm, nprob, s, count);
    case 256: return launch_batched<256>(B, prm, nprob, s, count);
    default: return launch_batched<512>(B, prm, nprob, s, count);
  }
}

b200::BParams batch_params(b200_batch B) {
  b200::BParams p{};
  p.nev = B->nev;
  p.ncv = B->ncv;
  p.mpd = B->mpd;
  p.max_it_user = B->max_it;
  p.which = B->which;
  p.tol = B->tol;
  p.eta = 0.7071;
  p.keep = 0.5;
  p.seed = 0x5eedULL;
  return p;
}

}  // namespace
}  // namespace b200

extern "C" b200_status b200_batch_create(int nprob, const int *ns, const int *rowptr, const int *colind,
                                         const double *vals, void *stream, b200_batch *out) {
  B200_ARG_CHECK(out && nprob > 0 && ns && rowptr && colind && vals, "invalid batch arguments");
  b200_batch B = new b200_batch_s;
  B->stream = (cudaStream_t)stream;
  B->nprob = nprob;
  B->ns.assign(ns, ns + nprob);
  // host plan: offsets and warp tiles of every problem
  std::vector<int4> tiles;
  long long rp = 0, nz = 0, rows = 0;
  B->hprobs.resize(nprob);
  for (int p = 0; p < nprob; ++p) {
    const int n = ns[p];
    if (n <= 0) {
      delete B;
      b200_set_last_error(__FILE__, __LINE__, "every problem needs at least one row");
      return B200_ERR_ARG;
    }
    const int *r = rowptr + rp;
    if (r[0] != 0) {
      delete B;
      b200_set_last_error(__FILE__, __LINE__, "every problem's row pointer must start at 0");
      return B200_ERR_ARG;
    }
    for (int i = 0; i < n; ++i)
      if (r[i + 1] < r[i] || r[i + 1] - r[i] > kWarpTileNnz) {
        delete B;
        b200_set_last_error(__FILE__, __LINE__, "batched rows need 0..256 nonzeros each");
        return B200_ERR_ARG;
      }
    for (int q = 0; q < r[n]; ++q)
      if (colind[nz + q] < 0 || colind[nz + q] >= n) {
        delete B;
        b200_set_last_error(__FILE__, __LINE__, "column index out of range");
        return B200_ERR_ARG;
      }
    WarpTiles wt = spmv_warp_tiles(n, r);
    b200::BProblem &P = B->hprobs[p];
    P.rp_off = rp;
    P.nnz_off = nz;
    P.tile_off = (long long)tiles.size();
    P.x_off = rows;
    P.nnz = r[n];
    P.n = n;
    P.ld = (n + 3) & ~3;
    P.ntiles = (int)wt.tiles.size();
    P.index = p;
    tiles.insert(tiles.end(), wt.tiles.begin(), wt.tiles.end());
    rp += n + 1;
    nz += r[n];
    rows += n;
  }
  B->total_rows = rows;
  std::vector<int> order(nprob);
  for (int p = 0; p < nprob; ++p) order[p] = p;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return ns[a] > ns[b]; });
  cudaStream_t s = B->stream;
  bool ok = cudaMalloc(&B->rowptr, sizeof(int) * rp) == cudaSuccess &&
            cudaMalloc(&B->colind, sizeof(int) * (nz > 0 ? nz : 1)) == cudaSuccess &&
            cudaMalloc(&B->vals, sizeof(double) * (nz > 0 ? nz : 1)) == cudaSuccess &&
            cudaMalloc(&B->tiles, sizeof(int4) * (tiles.empty() ? 1 : tiles.size())) == cudaSuccess &&
            cudaMalloc(&B->v0, sizeof(double) * rows) == cudaSuccess &&
            cudaMalloc(&B->order, sizeof(int) * nprob) == cudaSuccess &&
            cudaMalloc(&B->next, sizeof(int)) == cudaSuccess &&
            cudaMalloc(&B->probs, sizeof(b200::BProblem) * nprob) == cudaSuccess &&
            cudaMalloc(&B->info, sizeof(int) * 8 * nprob) == cudaSuccess &&
            cudaMalloc(&B->bytes, sizeof(double) * nprob) == cudaSuccess;
  if (ok) {
    ok = cudaMemcpyAsync(B->rowptr, rowptr, sizeof(int) * rp, cudaMemcpyHostToDevice, s) == cudaSuccess &&
         (nz == 0 || cudaMemcpyAsync(B->colind, colind, sizeof(int) * nz, cudaMemcpyHostToDevice, s) == cudaSuccess) &&
         (nz == 0 || cudaMemcpyAsync(B->vals, vals, sizeof(double) * nz, cudaMemcpyHostToDevice, s) == cudaSuccess) &&
         (tiles.empty() ||
          cudaMemcpyAsync(B->tiles, tiles.data(), sizeof(int4) * tiles.size(), cudaMemcpyHostToDevice, s) ==
              cudaSuccess) &&
         cudaMemcpyAsync(B->order, order.data(), sizeof(int) * nprob, cudaMemcpyHostToDevice, s) == cudaSuccess &&
         cudaMemsetAsync(B->v0, 0, sizeof(double) * rows, s) == cudaSuccess &&
         cudaStreamSynchronize(s) == cudaSuccess;
  }
  if (!ok) {
    b200_batch_destroy(B);
    b200_set_last_error(__FILE__, __LINE__, "device allocation or copy failed for the batch");
    return B200_ERR_NOMEM;
  }
  *out = B;
  return B200_OK;
}

extern "C" b200_status b200_batch_destroy(b200_batch B) {
  if (!B) return B200_OK;
  if (B->exec) cudaGraphExecDestroy(B->exec);
  if (B->graph) cudaGraphDestroy(B->graph);
  cudaFree(B->probs);
  cudaFree(B->rowptr);
  cudaFree(B->colind);
  cudaFree(B->vals);
  cudaFree(B->tiles);
  cudaFree(B->v0);
  cudaFree(B->V);
  cudaFree(B->order);
  cudaFree(B->next);
  cudaFree(B->evals);
  cudaFree(B->errest);
  cudaFree(B->vcol);
  cudaFree(B->info);
  cudaFree(B->bytes);
  cudaFree(B->V32);
  cudaFree(B->W);
  cudaFree(B->v0_2);
  cudaFree(B->info1);
  cudaFree(B->bytes1);
  delete B;
  return B200_OK;
}

extern "C" b200_status b200_batch_set_precision(b200_batch B, int precision, double tol_low) {
  B200_ARG_CHECK(B && (precision == B200_PRECISION_FP64 || precision == B200_PRECISION_MIXED), "unknown precision");
  B->precision = precision;
  B->tol_low = tol_low > 0.0 ? tol_low : 1e-6;
  B->solved = false;
  return B200_OK;
}

extern "C" b200_status b200_batch_set_dimensions(b200_batch B, int nev, int ncv, int mpd) {
  B200_ARG_CHECK(B && nev > 0, "nev must be positive");
  int n_min = *std::min_element(B->ns.begin(), B->ns.end());
  if (ncv <= 0) ncv = std::max(2 * nev, nev + 15);
  if (mpd <= 0) mpd = ncv;
  B200_ARG_CHECK(ncv >= nev + 1 && ncv + 1 <= 32, "batched: need nev < ncv <= 31");
  B200_ARG_CHECK(ncv <= n_min, "ncv cannot exceed the smallest problem size");
  B200_ARG_CHECK(ncv <= nev + mpd, "the value of ncv must not be larger than nev+mpd");
  B->nev = nev;
  B->ncv = ncv;
  B->mpd = mpd;
  B->solved = false;
  return B200_OK;
}

extern "C" b200_status b200_batch_set_tolerances(b200_batch B, double tol, int max_it) {
  B200_ARG_CHECK(B, "null argument");
  B->tol = tol > 0.0 ? tol : 1e-8;
  B->max_it = max_it > 0 ? max_it : 0;
  return B200_OK;
}

extern "C" b200_status b200_batch_set_which_eigenpairs(b200_batch B, int which) {
  B200_ARG_CHECK(B && which >= B200_LARGEST_MAGNITUDE && which <= B200_SMALLEST_REAL, "unsupported which");
  B->which = which;
  return B200_OK;
}

extern "C" b200_status b200_batch_set_initial_vectors(b200_batch B, const double *v0) {
  B200_ARG_CHECK(B && v0, "null argument");
  B200_CUDA_CHECK(cudaMemcpyAsync(B->v0, v0, sizeof(double) * B->total_rows, cudaMemcpyHostToDevice, B->stream));
  B200_CUDA_CHECK(cudaStreamSynchronize(B->stream));
  return B200_OK;
}

extern "C" b200_status b200_batch_set_threads(b200_batch B, int threads) {
  B200_ARG_CHECK(B && (threads == 0 || threads == 128 || threads == 256 || threads == 512),
                 "threads per problem must be 0 (autotune), 128, 256 or 512");
  B->threads = threads;
  return B200_OK;
}

static b200_status batch_alloc_mixed(b200_batch B) {
  if (B->precision != B200_PRECISION_MIXED || B->V32) return B200_OK;
  B200_CUDA_CHECK(cudaMalloc(&B->V32, sizeof(float) * (B->v_total ? B->v_total : 1)));
  B200_CUDA_CHECK(cudaMalloc(&B->W, sizeof(double) * B->total_rows));
  B200_CUDA_CHECK(cudaMalloc(&B->v0_2, sizeof(double) * B->total_rows));
  B200_CUDA_CHECK(cudaMalloc(&B->info1, sizeof(int) * 8 * (size_t)B->nprob));
  B200_CUDA_CHECK(cudaMalloc(&B->bytes1, sizeof(double) * B->nprob));
  return B200_OK;
}

static b200_status batch_alloc(b200_batch B) {
  if (B->ncv == 0) B200_CHECK(b200_batch_set_dimensions(B, B->nev, 0, 0));
  if (B->V && B->alloc_ncv == B->ncv) return batch_alloc_mixed(B);
  cudaFree(B->V32);  // sized with the bases
  B->V32 = nullptr;
  if (B->exec) cudaGraphExecDestroy(B->exec);
  if (B->graph) cudaGraphDestroy(B->graph);
  B->exec = nullptr;
  B->graph = nullptr;
  size_t total = 0;
  for (auto &P : B->hprobs) {
    P.v_off = (long long)total;
    total += (size_t)P.ld * (B->ncv + 1);
  }
  cudaFree(B->V);
  cudaFree(B->evals);
  cudaFree(B->errest);
  cudaFree(B->vcol);
  B->V = nullptr;
  B->evals = nullptr;
  B->errest = nullptr;
  B->vcol = nullptr;
  B200_CUDA_CHECK(cudaMalloc(&B->V, sizeof(double) * total));
  B->v_total = total;
  B200_CUDA_CHECK(cudaMalloc(&B->evals, sizeof(double) * (size_t)B->nprob * B->ncv));
  B200_CUDA_CHECK(cudaMalloc(&B->errest, sizeof(double) * (size_t)B->nprob * B->ncv));
  B200_CUDA_CHECK(cudaMalloc(&B->vcol, sizeof(int) * (size_t)B->nprob * B->ncv));
  B200_CUDA_CHECK(cudaMemcpyAsync(B->probs, B->hprobs.data(), sizeof(b200::BProblem) * B->nprob,
                                  cudaMemcpyHostToDevice, B->stream));
  B200_CUDA_CHECK(cudaStreamSynchronize(B->stream));
  B->alloc_ncv = B->ncv;
  return batch_alloc_mixed(B);
}

// Project-written autotuner: each candidate CTA size solves the largest problems of the batch
// (two waves of resident CTAs) and the fastest is kept.
extern "C" b200_status b200_batch_autotune(b200_batch B, int *threads_out) {
  B200_ARG_CHECK(B, "null argument");
  B200_CHECK(batch_alloc(B));
  const b200::BParams prm = batch_params(B);
  const int cands[3] = {128, 256, 512};
  cudaEvent_t e0, e1;
  B200_CUDA_CHECK(cudaEventCreate(&e0));
  B200_CUDA_CHECK(cudaEventCreate(&e1));
  float best = 1e30f;
  int best_t = 256;
  for (int t : cands) {
    int per_sm = 0;
    if (t == 128) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batched_ks_kernel<128>, 128, 0);
    else if (t == 256) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batched_ks_kernel<256>, 256, 0);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batched_ks_kernel<512>, 512, 0);
    const int sample = std::min(B->nprob, 2 * num_sms_host() * std::max(per_sm, 1));
    B200_CUDA_CHECK(cudaEventRecord(e0, B->stream));
    B200_CUDA_CHECK(launch_any(B, t, prm, sample, B->stream, true));
    B200_CUDA_CHECK(cudaEventRecord(e1, B->stream));
    B200_CUDA_CHECK(cudaEventSynchronize(e1));
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    // normalise by the rows solved so that candidates with different sample sizes compare
    std::vector<int> ord(B->nprob);
    for (int p = 0; p < B->nprob; ++p) ord[p] = p;
    std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return B->ns[a] > B->ns[b]; });
    double rows = 0;
    for (int i = 0; i < sample; ++i) rows += B->ns[ord[i]];
    const float per_row = (float)(ms / rows);
    if (per_row < best) {
      best = per_row;
      best_t = t;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  B->threads = best_t;
  if (threads_out) *threads_out = best_t;
  return B200_OK;
}

extern "C" b200_status b200_batch_solve(b200_batch B) {
  B200_ARG_CHECK(B, "null argument");
  B200_CHECK(batch_alloc(B));
  if (B->threads == 0) B200_CHECK(b200_batch_autotune(B, nullptr));
  const b200::BParams prm = batch_params(B);
  // one persistent launch (counter reset + kernel), captured once in a CUDA graph and replayed
  // while the launch shape, the parameters and the buffers stay the same
  const bool mixed = B->precision == B200_PRECISION_MIXED;
  if (!B->exec || B->graph_threads != B->threads || memcmp(&B->graph_prm, &prm, sizeof(prm)) != 0 ||
      B->graph_precision != B->precision || B->graph_tol_low != B->tol_low) {
    if (B->exec) cudaGraphExecDestroy(B->exec);
    if (B->graph) cudaGraphDestroy(B->graph);
    B->exec = nullptr;
    B->graph = nullptr;
    cudaStream_t cap = nullptr;
    B200_CUDA_CHECK(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    B200_CUDA_CHECK(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = mixed ? launch_mixed_any(B, B->threads, prm, cap, false)  // counted at each replay
                          : launch_any(B, B->threads, prm, B->nprob, cap, false);
    cudaGraph_t g = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(cap, &g);
    cudaStreamDestroy(cap);
    B200_CUDA_CHECK(e);
    B200_CUDA_CHECK(e2);
    B->graph = g;
    B200_CUDA_CHECK(cudaGraphInstantiate(&B->exec, g, 0));
    B->graph_threads = B->threads;
    B->graph_prm = prm;
    B->graph_precision = B->precision;
    B->graph_tol_low = B->tol_low;
  }
  cudaEvent_t e0, e1;
  B200_CUDA_CHECK(cudaEventCreate(&e0));
  B200_CUDA_CHECK(cudaEventCreate(&e1));
  B200_CUDA_CHECK(cudaEventRecord(e0, B->stream));
  B200_CUDA_CHECK(cudaGraphLaunch(B->exec, B->stream));
  count_launch();  // the graph holds one kernel (three in the mixed form)
  if (mixed) {
    count_launch();
    count_launch();
  }
  B200_CUDA_CHECK(cudaEventRecord(e1, B->stream));
  B200_CUDA_CHECK(cudaEventSynchronize(e1));
  cudaEventElapsedTime(&B->last_ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  B->h_evals.resize((size_t)B->nprob * B->ncv);
  B->h_errest.resize((size_t)B->nprob * B->ncv);
  B->h_vcol.resize((size_t)B->nprob * B->ncv);
  B->h_info.resize((size_t)B->nprob * 8);
  B200_CUDA_CHECK(cudaMemcpyAsync(B->h_evals.data(), B->evals, sizeof(double) * B->h_evals.size(),
                                  cudaMemcpyDeviceToHost, B->stream));
  B200_CUDA_CHECK(cudaMemcpyAsync(B->h_errest.data(), B->errest, sizeof(double) * B->h_errest.size(),
                                  cudaMemcpyDeviceToHost, B->stream));
  B200_CUDA_CHECK(
      cudaMemcpyAsync(B->h_vcol.data(), B->vcol, sizeof(int) * B->h_vcol.size(), cudaMemcpyDeviceToHost, B->stream));
  B200_CUDA_CHECK(
      cudaMemcpyAsync(B->h_info.data(), B->info, sizeof(int) * B->h_info.size(), cudaMemcpyDeviceToHost, B->stream));
  B->h_bytes.resize(B->nprob);
  B200_CUDA_CHECK(cudaMemcpyAsync(B->h_bytes.data(), B->bytes, sizeof(double) * B->nprob, cudaMemcpyDeviceToHost,
                                  B->stream));
  if (mixed) {
    B->h_info1.resize((size_t)B->nprob * 8);
    B->h_bytes1.resize(B->nprob);
    B200_CUDA_CHECK(cudaMemcpyAsync(B->h_info1.data(), B->info1, sizeof(int) * B->h_info1.size(),
                                    cudaMemcpyDeviceToHost, B->stream));
    B200_CUDA_CHECK(cudaMemcpyAsync(B->h_bytes1.data(), B->bytes1, sizeof(double) * B->nprob, cudaMemcpyDeviceToHost,
                                    B->stream));
  } else {
    B->h_info1.clear();
    B->h_bytes1.clear();
  }
  B200_CUDA_CHECK(cudaStreamSynchronize(B->stream));
  B->solved = true;
  for (int p = 0; p < B->nprob; ++p) {
    if (B->h_info[(size_t)p * 8] < 0) {
      b200_set_last_error(__FILE__, __LINE__, "a batched problem was not solved by the launch");
      return B200_ERR_DEVICE;
    }
    if (B->h_info[(size_t)p * 8 + 4]) {
      b200_set_last_error(__FILE__, __LINE__, "a batched problem reported a device-side error");
      return B200_ERR_DEVICE;
    }
  }
  B->solved = true;
  return B200_OK;
}

extern "C" b200_status b200_batch_get_solution(b200_batch B, int p, int *nconv, int *its, int *reason,
                                               int *lanczos_steps, double *evals, double *errest) {
  B200_ARG_CHECK(B && p >= 0 && p < B->nprob, "problem index out of range");
  if (!B->solved) {
    b200_set_last_error(__FILE__, __LINE__, "b200_batch_solve has not been called");
    return B200_ERR_STATE;
  }
  const int *inf = B->h_info.data() + (size_t)p * 8;
  if (nconv) *nconv = inf[0];
  if (its) *its = inf[1];
  if (reason) *reason = inf[2];
  if (lanczos_steps) *lanczos_steps = inf[3];
  for (int i = 0; i < std::min(inf[0], B->ncv); ++i) {
    if (evals) evals[i] = B->h_evals[(size_t)p * B->ncv + i];
    if (errest) errest[i] = B->h_errest[(size_t)p * B->ncv + i];
  }
  return B200_OK;
}

extern "C" b200_status b200_batch_get_eigenvector(b200_batch B, int p, int i, double *x_host) {
  B200_ARG_CHECK(B && p >= 0 && p < B->nprob && x_host, "invalid arguments");
  if (!B->solved) {
    b200_set_last_error(__FILE__, __LINE__, "b200_batch_solve has not been called");
    return B200_ERR_STATE;
  }
  const int nconv = B->h_info[(size_t)p * 8];
  B200_ARG_CHECK(i >= 0 && i < nconv, "eigenpair index out of range");
  const int c = B->h_vcol[(size_t)p * B->ncv + i];
  const b200::BProblem &P = B->hprobs[p];
  B200_CUDA_CHECK(cudaMemcpyAsync(x_host, B->V + P.v_off + (size_t)c * P.ld, sizeof(double) * P.n,
                                  cudaMemcpyDeviceToHost, B->stream));
  B200_CUDA_CHECK(cudaStreamSynchronize(B->stream));
  return B200_OK;
}

extern "C" b200_status b200_batch_get_all(b200_batch B, double *evals_host, int *info_host, float *ms) {
  B200_ARG_CHECK(B, "null argument");
  if (!B->solved) {
    b200_set_last_error(__FILE__, __LINE__, "b200_batch_solve has not been called");
    return B200_ERR_STATE;
  }
  if (evals_host) memcpy(evals_host, B->h_evals.data(), sizeof(double) * B->h_evals.size());
  if (info_host) memcpy(info_host, B->h_info.data(), sizeof(int) * B->h_info.size());
  if (ms) *ms = B->last_ms;
  return B200_OK;
}

extern "C" b200_status b200_batch_get_bytes(b200_batch B, double *bytes) {
  B200_ARG_CHECK(B && bytes, "null argument");
  if (!B->solved) {
    b200_set_last_error(__FILE__, __LINE__, "b200_batch_solve has not been called");
    return B200_ERR_STATE;
  }
  double t = 0.0;
  for (double b : B->h_bytes) t += b;
  for (double b : B->h_bytes1) t += b;  // phase 1 of the mixed form
  *bytes = t;
  return B200_OK;
}

extern "C" b200_status b200_batch_get_phase1(b200_batch B, int *info_host, double *bytes) {
  B200_ARG_CHECK(B, "null argument");
  if (!B->solved || B->h_info1.empty()) {
    b200_set_last_error(__FILE__, __LINE__, "no mixed-precision solve has run");
    return B200_ERR_STATE;
  }
  if (info_host) memcpy(info_host, B->h_info1.data(), sizeof(int) * B->h_info1.size());
  if (bytes) {
    double t = 0.0;
    for (double b : B->h_bytes1) t += b;
    *bytes = t;
  }
  return B200_OK;
}
